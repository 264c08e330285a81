"""ctypes access to the C restatement of the reference algorithm
(oracle/otmap_oracle.c, built into oracle/_build/liboracle.so by oracle/Makefile).

Test infrastructure only: the tests, __graft_entry__.smoke() and bench.py's
``cpu_baseline`` leg use it as the checker, never as the thing measured or shipped.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


class _Opts(C.Structure):
    _fields_ = [("beta_cj", C.c_int), ("max_iter", C.c_int), ("threshold", C.c_double),
                ("max_ratio", C.c_double)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"oracle not built: {LIB_PATH} (run make -C oracle oracle)")
        L = C.CDLL(LIB_PATH)
        L.oro_adjust_density.argtypes = [C.c_int, _dp, C.c_double]
        L.oro_vertex_gradients.argtypes = [C.c_int, _dp, _dp]
        L.oro_face_areas.argtypes = [C.c_int, _dp, _dp]
        L.oro_residual.argtypes = [C.c_int, _dp, _dp, _dp]
        L.oro_residual.restype = C.c_double
        L.oro_line_params.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
        L.oro_pick_step.argtypes = [_dp, _dp, _dp]
        L.oro_pick_step.restype = C.c_int
        L.oro_laplacian_apply.argtypes = [C.c_int, _dp, _dp]
        L.oro_poisson_dct.argtypes = [C.c_int, _dp, _dp]
        L.oro_poisson_pinned.argtypes = [C.c_int, _dp, _dp]
        L.oro_poisson_pinned.restype = C.c_int
        L.oro_solve.argtypes = [C.c_int, _dp, C.POINTER(_Opts), _dp, _dp, _dp, _dp, C.c_int, _dp]
        L.oro_solve.restype = C.c_int
        L.oro_apply_inverse.argtypes = [C.c_int, _dp, _dp, _dp, C.c_long, _ip, _ip]
        L.oro_apply_inverse.restype = C.c_long
        L.oro_bvh_build.argtypes = [C.c_int, _dp]
        L.oro_bvh_build.restype = C.c_void_p
        L.oro_bvh_free.argtypes = [C.c_void_p]
        L.oro_bvh_order.argtypes = [C.c_int, _dp, _ip, _dp]
        L.oro_bvh_query_all.argtypes = [C.c_void_p, _dp, C.c_int, _ip, _dp]
        L.oro_bvh_query_all.restype = C.c_int
        L.oro_bilinear_weights.argtypes = [_dp, _dp, _dp]
        L.oro_bilinear_weights.restype = C.c_int
        L.oro_inside_quad.argtypes = [_dp, _dp]
        L.oro_inside_quad.restype = C.c_int
        L.oro_rasterize.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_int, C.c_int, _dp]
        L.oro_transport_cost.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
        L.oro_transport_cost.restype = C.c_double
        L.oro_rasterize_mesh.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_int, _dp]
        L.oro_grid_faces.argtypes = [C.c_int, _ip, _ip]
        L.oro_mesh_blend.argtypes = [C.c_long, C.c_int, C.POINTER(_dp), _dp, _dp]
        L.oro_prune_empty_faces.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _dp, C.c_int, _ip, _dp, _ip, _ip, _ip]
        L.oro_prune_empty_faces.restype = C.c_int
        L.oro_grid_transport_cost.argtypes = [C.c_int, _dp, _dp, _dp]
        L.oro_grid_transport_cost.restype = C.c_double
        L.oro_sample_image.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _ip, C.c_ulonglong, C.c_int, C.c_int, _dp]
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_dp)


def adjust_density(density, max_ratio=np.finfo(np.float64).max):
    d = _f64(np.array(density, dtype=np.float64, copy=True))
    n = int(round(np.sqrt(d.size)))
    lib().oro_adjust_density(n, _p(d), float(max_ratio))
    return d


def vertex_gradients(psi, n):
    g = np.zeros(((n + 1) ** 2, 2))
    lib().oro_vertex_gradients(n, _p(_f64(psi)), _p(g))
    return g


def residual(psi, density, n):
    r = np.zeros(n * n)
    v = lib().oro_residual(n, _p(_f64(psi)), _p(_f64(density)), _p(r))
    return r, v


def line_params(g0, gd, n):
    a = np.zeros(n * n)
    b = np.zeros(n * n)
    lib().oro_line_params(n, _p(_f64(g0)), _p(_f64(gd)), _p(a), _p(b))
    return a, b


def pick_step(z):
    z = _f64(z)
    al = C.c_double(0)
    em = C.c_double(0)
    found = lib().oro_pick_step(_p(z), C.byref(al), C.byref(em))
    return al.value, em.value, bool(found)


def laplacian_apply(x, n):
    y = np.zeros(n * n)
    lib().oro_laplacian_apply(n, _p(_f64(x)), _p(y))
    return y


def poisson_dct(r, n):
    d = np.zeros(n * n)
    lib().oro_poisson_dct(n, _p(_f64(r)), _p(d))
    return d


def poisson_pinned(r, n):
    d = np.zeros(n * n)
    rc = lib().oro_poisson_pinned(n, _p(_f64(r)), _p(d))
    if rc != 0:
        raise RuntimeError("pinned Cholesky failed")
    return d


class Result:
    pass


def solve(density_cells, n, beta_cj=True, max_iter=1000, threshold=1e-7,
          max_ratio=np.finfo(np.float64).max, trace=True):
    """The whole solve (otsolver_2dgrid.cpp:106-245)."""
    d = _f64(density_cells)
    assert d.size == n * n
    opts = _Opts(int(bool(beta_cj)), int(max_iter), float(threshold), float(max_ratio))
    psi = np.zeros(n * n)
    fwd = np.zeros(((n + 1) ** 2, 2))
    dens = np.zeros(n * n)
    tr = np.zeros((max(max_iter, 1), 5))
    res = C.c_double(0)
    it = lib().oro_solve(n, _p(d), C.byref(opts), _p(psi), _p(fwd), _p(dens), _p(tr) if trace else None,
                         max_iter if trace else 0, C.byref(res))
    out = Result()
    out.n = n
    out.iterations = it
    out.residual = res.value
    out.psi = psi
    out.fwd = fwd
    out.density = dens
    out.trace = tr[:it].copy() if trace else None
    return out


def apply_inverse(fwd_xy, density, n, pts):
    """apply_inverse_map (transport_map.cpp:105-128): positions, chosen faces, hit counts."""
    p = _f64(np.array(pts, dtype=np.float64, copy=True))
    P = p.shape[0]
    faces = np.zeros(P, dtype=np.int32)
    nh = np.zeros(P, dtype=np.int32)
    missing = lib().oro_apply_inverse(n, _p(_f64(fwd_xy)), _p(_f64(density)), _p(p), P,
                                      faces.ctypes.data_as(_ip), nh.ctypes.data_as(_ip))
    return p, faces, nh, missing


def query_all(fwd_xy, n, pts, cap=4):
    """BVH2D::query_all hits (clamped points), traversal order."""
    fwd = _f64(fwd_xy)
    b = lib().oro_bvh_build(n, _p(fwd))
    pts = np.clip(_f64(pts), 0.0, 1.0)
    P = pts.shape[0]
    nh = np.zeros(P, dtype=np.int32)
    faces = np.full((P, cap), -1, dtype=np.int32)
    bary = np.zeros((P, cap, 4))
    fb = np.zeros(cap, dtype=np.int32)
    bb = np.zeros(4 * cap)
    for i in range(P):
        q = _f64(pts[i])
        k = lib().oro_bvh_query_all(b, _p(q), cap, fb.ctypes.data_as(_ip), _p(bb))
        nh[i] = k
        m = min(k, cap)
        faces[i, :m] = fb[:m]
        bary[i, :m] = bb[: 4 * m].reshape(m, 4)
    lib().oro_bvh_free(b)
    return nh, faces, bary


def rasterize(xy, n, density, rows, cols, stale_weights=True):
    img = np.zeros((rows, cols))
    d = None if density is None else _f64(density)
    lib().oro_rasterize(n, _p(_f64(xy)), None if d is None else _p(d), rows, cols,
                        int(bool(stale_weights)), _p(img))
    return img


def transport_cost(src_xy, dst_xy, density, n, per_face=False):
    pf = np.zeros(n * n) if per_face else None
    c = lib().oro_transport_cost(n, _p(_f64(src_xy)), _p(_f64(dst_xy)), _p(_f64(density)),
                                 None if pf is None else _p(pf))
    return (c, pf) if per_face else c


def grid_vertices(n):
    """Origin mesh vertices (i/n, j/n) in vertex order v = j + i*(n+1), AoS."""
    t = np.arange(n + 1, dtype=np.float64) * (1.0 / n)
    X = np.repeat(t, n + 1)
    Y = np.tile(t, n + 1)
    return np.stack([X, Y], axis=1)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _pi(a):
    return a.ctypes.data_as(_ip)


def grid_faces(n):
    """The (n+1)^2 grid's quads as (start[N+1], idx[4N]) in circulation order."""
    start = np.zeros(n * n + 1, dtype=np.int32)
    idx = np.zeros(4 * n * n, dtype=np.int32)
    lib().oro_grid_faces(n, _pi(start), _pi(idx))
    return start, idx


def rasterize_mesh(xy, start, idx, density, rows, cols, per_vertex=False, stale_weights=True):
    """rasterize_image on an indexed triangle/quad mesh; image is [y][x]."""
    xy = _f64(xy).reshape(-1, 2)
    start, idx = _i32(start), _i32(idx)
    img = np.zeros((rows, cols))
    d = None if density is None else _f64(density)
    lib().oro_rasterize_mesh(xy.shape[0], _p(xy), start.size - 1, _pi(start), _pi(idx),
                             None if d is None else _p(d), 0 if d is None else d.size, rows, cols,
                             0 if per_vertex else 1, int(bool(stale_weights)), _p(img))
    return img


def mesh_blend(meshes, weights):
    """out = sum_k weights[k] * meshes[k] (apps/barycenters.cpp:250-276)."""
    ms = [_f64(m) for m in meshes]
    w = _f64(weights)
    out = np.empty_like(ms[0])
    arr = (_dp * len(ms))(*[_p(m) for m in ms])
    lib().oro_mesh_blend(ms[0].size, len(ms), arr, _p(w), _p(out))
    return out


def prune_empty_faces(xy, start, idx, density):
    """prune_empty_faces + garbage collection -> (xy, start, idx)."""
    xy = _f64(xy).reshape(-1, 2)
    start, idx, d = _i32(start), _i32(idx), _f64(density)
    nv, nf = C.c_int(0), C.c_int(0)
    xo = np.zeros_like(xy)
    so = np.zeros_like(start)
    io = np.zeros_like(idx)
    lib().oro_prune_empty_faces(xy.shape[0], _p(xy), start.size - 1, _pi(start), _pi(idx), _p(d), d.size,
                                C.byref(nv), _p(xo), C.byref(nf), _pi(so), _pi(io))
    return xo[:nv.value].copy(), so[:nf.value + 1].copy(), io[:so[nf.value]].copy()


def sample_image(xy, start, idx, spf, seed, rows, cols):
    """Stochastic splat with the library's generator; image is [y][x]."""
    xy = _f64(xy).reshape(-1, 2)
    start, idx, spf = _i32(start), _i32(idx), _i32(spf)
    img = np.zeros((rows, cols))
    lib().oro_sample_image(xy.shape[0], _p(xy), start.size - 1, _pi(start), _pi(idx), _pi(spf), int(seed), rows,
                           cols, _p(img))
    return img


def grid_transport_cost(grads, density, n):
    """compute_transport_cost restated -> (sum, per-face costs)."""
    pf = np.zeros(n * n)
    c = lib().oro_grid_transport_cost(n, _p(_f64(grads)), _p(_f64(density)), _p(pf))
    return c, pf


def bvh_order(fwd_xy, n):
    """The reference BVH's final face array and each face's leaf box (bvh2d.cpp:29-64,
    167-242, with the (4, 24) of transport_map.cpp:40) -> (faces[pos], leaf_box[f, 4])."""
    N = n * n
    faces = np.zeros(N, dtype=np.int32)
    boxes = np.zeros((N, 4))
    lib().oro_bvh_order(int(n), _p(_f64(fwd_xy)), faces.ctypes.data_as(_ip), _p(boxes))
    return faces, boxes
