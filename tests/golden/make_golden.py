"""Regenerates the golden fixtures in this folder from the reference otmap library
compiled from its own sources (oracle/_ref/libotref.so, built by `make -C oracle ref`).

The reference ships no tests or fixtures, so these vectors are its own outputs on
seeded synthetic inputs (otmap_b200.workloads), small enough to commit:

  solve_*.npz     GridBasedTransportSolver::init/solve (otsolver_2dgrid.cpp:75-245):
                  input density, adjusted density, forward mesh, iterations, final
                  residual, per-iteration {alpha, beta, norm(d), res^2, Linf} trace
  inverse_*.npz   apply_inverse_map (transport_map.cpp:105-128) of grid vertices and
                  random points, and BVH2D::query_all hit lists (bvh2d.cpp:84-92)
  raster_*.npz    rasterize_image PerFace (rasterizer.cpp:188-236, :305-308)
  units_*.npz     protected solver steps on random potentials: vertex gradients,
                  residual, Laplacian solve, line-search coefficients, one line search
  cost_*.npz      transport_cost (transport_map.cpp:131-215)

Run:  python tests/golden/make_golden.py
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from otmap_b200 import workloads as W  # noqa: E402

DBL_MAX = np.finfo(np.float64).max


def grid_vertices(n):
    t = np.arange(n + 1, dtype=np.float64) * (1.0 / n)
    return np.stack([np.repeat(t, n + 1), np.tile(t, n + 1)], axis=1)


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name), **arrays)


SOLVE_CASES = [
    # name, n, density generator, options (beta_cj, max_iter, threshold, max_ratio)
    ("solve_mix_n16_s3", 16, lambda: W.gaussian_mixture(16, 3), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n32_s0", 32, lambda: W.gaussian_mixture(32, 0), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n64_s1", 64, lambda: W.gaussian_mixture(64, 1), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n128_s2", 128, lambda: W.gaussian_mixture(128, 2), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_shapes_n64_s5", 64, lambda: W.blurred_shapes(64, 5, sigma_px=1.5), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n48_s4_beta0", 48, lambda: W.gaussian_mixture(48, 4), (False, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n40_s6_ratio", 40, lambda: W.gaussian_mixture(40, 6, floor=1e-4), (True, 1000, 1e-7, 20.0)),
    ("solve_mix_n32_s7_iter5", 32, lambda: W.gaussian_mixture(32, 7), (True, 5, 1e-7, DBL_MAX)),
    ("solve_mix_n24_s8_th1e-4", 24, lambda: W.gaussian_mixture(24, 8), (True, 1000, 1e-4, DBL_MAX)),
    ("solve_const_n16", 16, lambda: np.ones((16, 16)), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n1", 1, lambda: np.ones((1, 1)), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n2_s9", 2, lambda: W.gaussian_mixture(2, 9), (True, 1000, 1e-7, DBL_MAX)),
    ("solve_mix_n37_s10", 37, lambda: W.gaussian_mixture(37, 10), (True, 1000, 1e-7, DBL_MAX)),
]


def main():
    s = ref.RefSolver()
    maps = {}
    for name, n, gen, (beta_cj, max_iter, th, ratio) in SOLVE_CASES:
        img = gen()
        d = W.to_cells(img)
        s.init(n)
        m = s.solve(d, beta_cj=beta_cj, max_iter=max_iter, threshold=th, max_ratio=ratio, trace=True)
        save(name + ".npz", n=n, density=d, adjusted=m.density(), fwd=m.fwd(),
             iterations=m.iterations, residual=m.residual, trace=m.trace,
             beta_cj=int(beta_cj), max_iter=max_iter, threshold=th, max_ratio=ratio)
        maps[name] = (n, m)
        print(name, "iters", m.iterations, "residual", m.residual)

    # inversion of grid vertices and random points on a few maps
    for name in ["solve_mix_n32_s0", "solve_mix_n64_s1", "solve_shapes_n64_s5", "solve_mix_n37_s10"]:
        n, m = maps[name]
        fwd = m.fwd()
        pts = np.concatenate([grid_vertices(n), W.random_points(2000, 7),
                              np.array([[-0.1, 0.5], [1.2, 0.3], [0.5, -1.0], [0.0, 0.0], [1.0, 1.0]])])
        inv, _ = m.apply_inverse(pts)
        nh, faces, bary = ref.query_all(fwd, n, pts, cap=4)
        # the forward mesh and density are those of the matching solve_*.npz fixture
        save("inverse_" + name[6:] + ".npz", n=n, solve=name, points=pts, inverse=inv, nhits=nh,
             faces=faces[:, :2], bary=bary[:, 0])
        print("inverse", name, "multi-hit", int((nh > 1).sum()), "no-hit", int((nh == 0).sum()))

    # rasterization of forward meshes (per-face density and unit density), square and ragged sizes
    for name in ["solve_mix_n32_s0", "solve_mix_n64_s1", "solve_shapes_n64_s5"]:
        n, m = maps[name]
        fwd = m.fwd()
        out = {"n": n, "solve": name}
        for tag, dn in [("dens", m.density()), ("unit", None)]:
            for rows, cols in [(n, n), (2 * n + 3, n + 5), (n // 2, n)]:
                img, _ = ref.rasterize(fwd, n, dn, rows, cols)
                out[f"img_{tag}_{rows}x{cols}"] = img
        save("raster_" + name[6:] + ".npz", **out)

    # protected steps on random potentials
    rng = np.random.default_rng(123)
    for n in (8, 31, 48):
        s.init(n)
        N = n * n
        dens = W.to_cells(W.gaussian_mixture(n, n))
        dens = dens / (dens.sum() / N)
        psi = rng.standard_normal(N) * 0.3 / (n * n)
        direc = rng.standard_normal(N) * 0.3 / (n * n)
        g = s.vertex_gradients(psi)
        r, res = s.residual(psi, dens)
        rc = r - r.mean()
        lap = s.laplacian_solve(rc)
        a, b = s.line_params(psi, direc)
        x1, r1, alpha, res1 = s.line_search(psi, direc, r, res)
        save(f"units_n{n}.npz", n=n, density=dens, psi=psi, direction=direc, grads=g, r=r, res=res,
             rhs=rc, lap=lap, a=a, b=b, psi1=x1, r1=r1, alpha=alpha, res1=res1)

    # transport cost origin -> forward mesh
    for name in ["solve_mix_n32_s0", "solve_shapes_n64_s5"]:
        n, m = maps[name]
        c, pf = ref.transport_cost(grid_vertices(n), m.fwd(), n, m.density(), per_face=True)
        save("cost_" + name[6:] + ".npz", n=n, solve=name, cost=c, per_face=pf)


if __name__ == "__main__":
    main()
