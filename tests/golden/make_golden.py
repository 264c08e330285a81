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
  rasterpv_*.npz  rasterize_image RIO_PerVertexDensity on the grid (rasterizer.cpp:237-302)
  meshraster_*.npz  rasterize_image on a triangulated grid and on a pruned quad mesh,
                  both options, and the pruned meshes themselves (mesh_utils.cpp:124-141)
  barycenter_*.npz  apps/barycenters.cpp:250-290 on four (and two) solved densities:
                  inverse meshes, blended meshes, rescaled images, expected means
  compose_*.npz   apps/otmap.cpp:120-137: composite maps u->v, v->u and their costs

Run:  python tests/golden/make_golden.py [group ...]   (groups: base extra; default both)
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


def solve_all():
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
    return s, maps


def base_fixtures(s, maps):

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


def triangulate(idx):
    """Each grid quad (v0, v1, v2, v3) as the triangles (v0, v1, v2), (v0, v2, v3)."""
    q = idx.reshape(-1, 4)
    tri = np.stack([q[:, [0, 1, 2]], q[:, [0, 2, 3]]], 1).reshape(-1).astype(np.int32)
    return np.arange(0, tri.size + 1, 3, dtype=np.int32), tri


def extra_fixtures(s, maps):
    from oracle import port

    # PerVertex raster of the grid forward meshes
    for name in ["solve_mix_n32_s0", "solve_mix_n64_s1", "solve_shapes_n64_s5"]:
        n, m = maps[name]
        out = {"n": n, "solve": name}
        for tag, dn in [("dens", m.density()), ("unit", None)]:
            for rows, cols in [(n, n), (2 * n + 3, n + 5), (n // 2, n)]:
                img, _ = ref.rasterize(m.fwd(), n, dn, rows, cols, per_vertex=True)
                out[f"img_{tag}_{rows}x{cols}"] = img
        save("rasterpv_" + name[6:] + ".npz", **out)

    # triangulated grid and pruned meshes, both options
    rng = np.random.default_rng(5)
    for name in ["solve_mix_n32_s0", "solve_shapes_n64_s5"]:
        n, m = maps[name]
        st, ix = port.grid_faces(n)
        tst, tix = triangulate(ix)
        dz = m.density().copy()
        dz[rng.random(dz.size) < 0.25] = 0
        dz[: n * 2] = 0
        pxy, pst, pix = ref.prune_empty_faces(m.fwd(), st, ix, dz)
        txy, tst2, tix2 = ref.prune_empty_faces(m.fwd(), tst, tix, dz)
        out = {"n": n, "solve": name, "zeroed": dz, "tri_start": tst, "tri_idx": tix, "pruned_xy": pxy,
               "pruned_start": pst, "pruned_idx": pix, "tpruned_xy": txy, "tpruned_start": tst2,
               "tpruned_idx": tix2}
        rows, cols = n + 3, n - 2
        for mode, pv in [("face", False), ("vertex", True)]:
            out[f"tri_dens_{mode}"] = ref.rasterize_mesh(m.fwd(), tst, tix, np.repeat(m.density(), 2), rows, cols,
                                                         per_vertex=pv)
            out[f"tri_unit_{mode}"] = ref.rasterize_mesh(m.fwd(), tst, tix, None, rows, cols, per_vertex=pv)
            out[f"pruned_unit_{mode}"] = ref.rasterize_mesh(pxy, pst, pix, None, rows, cols, per_vertex=pv)
            out[f"tpruned_unit_{mode}"] = ref.rasterize_mesh(txy, tst2, tix2, None, rows, cols, per_vertex=pv)
        save("meshraster_" + name[6:] + ".npz", **out)

    # bilinear and linear barycenters of four blurred-shape densities at 32^2
    n = 32
    imgs = [W.blurred_shapes(n, 40 + k, sigma_px=1.0) for k in range(4)]
    inv, fwd, adj, means = [], [], [], []
    s.init(n)
    for img in imgs:
        m = s.solve(W.to_cells(img))
        fwd.append(m.fwd())
        adj.append(m.density())
        q, _ = m.apply_inverse(grid_vertices(n))
        inv.append(q)
        means.append(ref.image_mean(img))
    out = {"n": n, "images": np.stack(imgs), "fwd": np.stack(fwd), "adjusted": np.stack(adj), "inv": np.stack(inv),
           "means": np.array(means)}
    pairs = [(0.0, 0.0), (0.25, 0.5), (0.75, 0.25), (0.5, 0.5), (1.0, 1.0), (1.0, 0.0)]
    out["pairs"] = np.array(pairs)
    for k, (a, b) in enumerate(pairs):
        mesh, img, e = ref.barycenter(n, inv, a, b, means, n, n)
        out[f"mesh_{k}"], out[f"img_{k}"], out[f"expected_{k}"] = mesh, img, e
    for k, a in enumerate([0.0, 0.3, 1.0]):
        mesh, img, e = ref.barycenter(n, inv[:2], a, 0.0, means[:2], n, n)
        out[f"lmesh_{k}"], out[f"limg_{k}"], out[f"lexpected_{k}"] = mesh, img, e
    out["lalphas"] = np.array([0.0, 0.3, 1.0])
    save("barycenter_shapes_n32.npz", **out)

    # composite maps between two solves of different sizes (apps/otmap.cpp:120-137)
    nu, mu = maps["solve_mix_n32_s0"]
    nv, mv = maps["solve_mix_n37_s10"]
    uv, _ = mv.apply_inverse(mu.fwd())
    vu, _ = mu.apply_inverse(mv.fwd())
    nh_uv, _, _ = ref.query_all(mv.fwd(), nv, np.clip(mu.fwd(), 0, 1), cap=4)
    nh_vu, _, _ = ref.query_all(mu.fwd(), nu, np.clip(mv.fwd(), 0, 1), cap=4)
    c_uv = ref.transport_cost(grid_vertices(nu), uv, nu, mu.density())
    c_vu = ref.transport_cost(grid_vertices(nv), vu, nv, mv.density())
    save("compose_mix_n32_n37.npz", u="solve_mix_n32_s0", v="solve_mix_n37_s10", map_uv=uv, map_vu=vu,
         nhits_uv=nh_uv, nhits_vu=nh_vu, cost_uv=c_uv, cost_vu=c_vu)
    print("compose: multi-hit", int((nh_uv > 1).sum()), int((nh_vu > 1).sum()))

    # the solver's quadrature transport cost (otsolver_2dgrid.cpp:608-640)
    for name in ["solve_mix_n32_s0", "solve_shapes_n64_s5"]:
        n, m = maps[name]
        s.init(n)
        grads = m.fwd() - grid_vertices(n)
        total, pf = s.grid_transport_cost(grads, m.density())
        save("gridcost_" + name[6:] + ".npz", n=n, solve=name, grads=grads, total=total, per_face=pf)


def main(groups):
    s, maps = solve_all()
    if "base" in groups:
        base_fixtures(s, maps)
    if "extra" in groups:
        extra_fixtures(s, maps)


if __name__ == "__main__":
    main(sys.argv[1:] or ["base", "extra"])
