"""Builds tests/cpp/facade_demo.cpp (the C++ facade's test driver) against the
in-tree library; shared by the CPU and GPU facade tests."""

import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "facade_demo.cpp")


def cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")


def build(out_dir, eigen_include=None):
    from otmap_b200 import build as B

    if not os.path.exists(B.LIB):
        B.build_library()
    exe = os.path.join(out_dir, "facade_demo" + ("_eigen" if eigen_include else ""))
    cmd = [cxx(), "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", B.INCLUDE, SRC, "-L", B.LIBDIR, "-lotmap_b200",
           "-Wl,-rpath," + B.LIBDIR, "-o", exe]
    if eigen_include:
        cmd[4:4] = ["-isystem", eigen_include]
    else:
        cmd.insert(4, "-DOTMAP_B200_NO_EIGEN")
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    return exe


def results(folder):
    out = {}
    with open(os.path.join(folder, "results.txt")) as f:
        for line in f:
            k, v = line.split()
            out[k] = float(v)
    return out
