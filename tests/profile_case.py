"""A short, fixed solve for kernel profiling (ncu) and quick timing.

    python tests/profile_case.py [--n 1024] [--batch 2] [--iters 3] [--poisson fft|dense|tensor] [--precision fp64|split]

Solves `batch` blurred-shape densities of size n for a fixed number of iterations
(max_iter = iters, so every instance runs exactly that many) through the C ABI, with
inputs and outputs already on the device, and prints per-kernel CUDA-event times.
Small enough for a full ncu capture: the device holds batch * 11 * n^2 doubles.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--batch", type=int, default=2)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--poisson", default="fft", choices=["fft", "dense", "tensor"])
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "split"])
    a = ap.parse_args()

    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    ctx = N.Context(0)
    ctx.set_poisson({"fft": N.POISSON_FFT, "dense": N.POISSON_DENSE, "tensor": N.POISSON_TENSOR}[a.poisson])
    ctx.set_precision(N.PRECISION_SPLIT if a.precision == "split" else N.PRECISION_FP64)
    n, B = a.n, a.batch
    dens = [torch.from_numpy(W.to_cells(W.blurred_shapes(n, k, sigma_px=5.0))).cuda() for k in range(B)]
    fwd = [torch.empty(((n + 1) ** 2, 2), dtype=torch.float64, device="cuda") for _ in range(B)]
    opt = N.default_options()
    opt.max_iter = a.iters
    opt.threshold = 0.0
    stats = (N.SolveStatsC * B)()
    ns = (C.c_int * B)(*([n] * B))
    dp = (C.c_void_p * B)(*[d.data_ptr() for d in dens])
    fp = (C.c_void_p * B)(*[f.data_ptr() for f in fwd])
    ctx.init(n)
    ctx.profile(1)
    for _ in range(a.repeat):
        N.check(N.lib().otm_solve_batch(ctx.handle, B, ns, dp, C.byref(opt), fp, None, stats))
    prof = ctx.profile_totals()
    ctx.profile(0)
    out = {k: {"ms": v[0], "launches": v[1], "us_per_launch": 1e3 * v[0] / max(v[1], 1)} for k, v in prof.items()}
    print(json.dumps({"n": n, "batch": B, "iters": [stats[k].iterations for k in range(B)], "kernels": out}))
    ctx.close()


if __name__ == "__main__":
    main()
