"""Builds the CUDA library in-tree: otmap_b200/lib/libotmap_b200.so (sm_100a).

    python -m otmap_b200.build            # library only

nvcc cross-compiles for sm_100a without a GPU. The host compiler is pinned to the
system g++ so the library links the system libstdc++ dynamically (a statically
linked copy would clash with the one already loaded by Python/torch).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libotmap_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["capi.cu", "solver.cu", "stencil.cu", "poisson.cu", "dct_reg.cu", "dct_tc.cu", "adjoint.cu", "locate.cu",
           "pipeline.cu", "meshio.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _run(cmd):
    r = subprocess.run(cmd, cwd=ROOT, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("command failed: " + " ".join(cmd))
    return r.stdout


def build_library(verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    # no FMA contraction: per-cell arithmetic and the geometric predicates round as the
    # reference's scalar code does; kernels that want FMAs call fma() explicitly
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-fmad=false", "--expt-relaxed-constexpr",
           "-ccbin", host_cxx(), "-Xcompiler", "-fPIC", "-shared", "-I", INCLUDE, "-o", LIB, *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    out = _run(cmd)
    if verbose:
        sys.stdout.write(out)
    return LIB


if __name__ == "__main__":
    build_library(verbose="-v" in sys.argv)
    print(LIB)
