"""ctypes access to the reference otmap library built from its own sources
(oracle/_ref/libotref.so, see oracle/Makefile and oracle/ref_driver.cpp).

Test infrastructure only: used by the tests, the golden-fixture generator and the
CPU arm of bench.py as the checker and the timed CPU baseline, never by the product.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libotref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"reference library not built: {LIB_PATH} (run make -C oracle ref)")
        L = C.CDLL(LIB_PATH)
        L.otref_solver_new.restype = C.c_void_p
        L.otref_solver_free.argtypes = [C.c_void_p]
        L.otref_solver_init.argtypes = [C.c_void_p, C.c_int]
        L.otref_solver_init.restype = C.c_double
        L.otref_solve.argtypes = [C.c_void_p, _dp, C.c_int, C.c_int, C.c_double, C.c_double,
                                  _dp, C.c_int, _ip, _dp, _dp]
        L.otref_solve.restype = C.c_void_p
        L.otref_map_free.argtypes = [C.c_void_p]
        L.otref_map_fwd.argtypes = [C.c_void_p, _dp]
        L.otref_map_density.argtypes = [C.c_void_p, _dp]
        L.otref_apply_inverse.argtypes = [C.c_void_p, _dp, C.c_long]
        L.otref_apply_inverse.restype = C.c_double
        L.otref_query_all.argtypes = [_dp, C.c_int, _dp, C.c_long, C.c_int, _ip, _ip, _dp]
        L.otref_rasterize.argtypes = [_dp, C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp]
        L.otref_rasterize.restype = C.c_double
        L.otref_transport_cost.argtypes = [_dp, _dp, C.c_int, _dp, _dp]
        L.otref_transport_cost.restype = C.c_double
        L.otref_vertex_gradients.argtypes = [C.c_void_p, _dp, _dp]
        L.otref_residual.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.otref_residual.restype = C.c_double
        L.otref_laplacian_solve.argtypes = [C.c_void_p, _dp, _dp]
        L.otref_1d_params.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.otref_line_search.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp]
        L.otref_line_search.restype = C.c_double
        L.otref_rasterize_mesh.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _dp, C.c_int, C.c_int, C.c_int,
                                           C.c_int, _dp]
        L.otref_rasterize_mesh.restype = C.c_double
        L.otref_barycenter.argtypes = [C.c_int, C.c_int, C.POINTER(_dp), C.c_double, C.c_double, _dp, C.c_int,
                                       C.c_int, _dp, _dp]
        L.otref_barycenter.restype = C.c_double
        L.otref_image_mean.argtypes = [_dp, C.c_int, C.c_int]
        L.otref_image_mean.restype = C.c_double
        L.otref_prune.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _dp, C.c_int, _ip, _dp, _ip, _ip, _ip]
        L.otref_write_off.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, C.c_char_p]
        L.otref_write_off.restype = C.c_int
        L.otref_read_off.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _ip, _dp, _ip, _ip, _ip]
        L.otref_read_off.restype = C.c_int
        L.otref_grid_transport_cost.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.otref_grid_transport_cost.restype = C.c_double
        L.otref_sample_image.argtypes = [C.c_int, _dp, C.c_int, _ip, _ip, _ip, C.c_uint, C.c_int, C.c_int, _dp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class RefSolver:
    """otmap::GridBasedTransportSolver (otlib/otsolver_2dgrid.h:45-125)."""

    def __init__(self):
        self._h = lib().otref_solver_new()
        self.n = None
        self.init_seconds = 0.0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().otref_solver_free(self._h)
            self._h = None

    def init(self, n: int) -> float:
        self.init_seconds = lib().otref_solver_init(self._h, int(n))
        self.n = int(n)
        return self.init_seconds

    def solve(self, density_cells, beta_cj=True, max_iter=1000, threshold=1e-7,
              max_ratio=np.finfo(np.float64).max, trace=False):
        d = _f64(density_cells)
        assert d.size == self.n * self.n
        cap = max_iter if trace else 0
        tr = np.zeros((max(cap, 1), 5))
        it = C.c_int(0)
        res = C.c_double(0)
        sec = C.c_double(0)
        h = lib().otref_solve(self._h, _p(d), int(bool(beta_cj)), int(max_iter), float(threshold),
                              float(max_ratio), _p(tr) if trace else None, cap, C.byref(it),
                              C.byref(res), C.byref(sec))
        m = RefMap(h, self.n)
        m.iterations = it.value
        m.residual = res.value
        m.seconds = sec.value
        m.trace = tr[: it.value].copy() if trace else None
        return m

    # unit probes of the solver's protected steps
    def grid_transport_cost(self, grads, density):
        """compute_transport_cost (otsolver_2dgrid.cpp:608-640) -> (sum, per-face costs)."""
        pf = np.zeros(self.n * self.n)
        c = lib().otref_grid_transport_cost(self._h, _p(_f64(grads)), _p(_f64(density)), _p(pf))
        return c, pf

    def vertex_gradients(self, psi):
        g = np.zeros(((self.n + 1) ** 2, 2))
        lib().otref_vertex_gradients(self._h, _p(_f64(psi)), _p(g))
        return g

    def residual(self, psi, density):
        r = np.zeros(self.n * self.n)
        v = lib().otref_residual(self._h, _p(_f64(psi)), _p(_f64(density)), _p(r))
        return r, v

    def laplacian_solve(self, r):
        d = np.zeros(self.n * self.n)
        lib().otref_laplacian_solve(self._h, _p(_f64(r)), _p(d))
        return d

    def line_params(self, psi, direction):
        a = np.zeros(self.n * self.n)
        b = np.zeros(self.n * self.n)
        lib().otref_1d_params(self._h, _p(_f64(psi)), _p(_f64(direction)), _p(a), _p(b))
        return a, b

    def line_search(self, psi, direction, r, ek):
        N = self.n * self.n
        x1 = np.zeros(N)
        r1 = np.zeros(N)
        al = C.c_double(0)
        res = lib().otref_line_search(self._h, _p(_f64(psi)), _p(_f64(direction)), _p(_f64(r)),
                                      float(ek), _p(x1), _p(r1), C.byref(al))
        return x1, r1, al.value, res


class RefMap:
    """otmap::TransportMap (otlib/transport_map.h:29-63)."""

    def __init__(self, h, n):
        self._h = h
        self.n = n

    def __del__(self):
        if getattr(self, "_h", None):
            lib().otref_map_free(self._h)
            self._h = None

    def fwd(self):
        xy = np.zeros(((self.n + 1) ** 2, 2))
        lib().otref_map_fwd(self._h, _p(xy))
        return xy

    def density(self):
        d = np.zeros(self.n * self.n)
        lib().otref_map_density(self._h, _p(d))
        return d

    def apply_inverse(self, pts):
        p = _f64(np.array(pts, dtype=np.float64, copy=True))
        sec = lib().otref_apply_inverse(self._h, _p(p), p.shape[0])
        return p, sec


def query_all(fwd_xy, n, pts, cap=4):
    """BVH2D::query_all hits per point (otlib/utils/bvh2d.cpp:84-92)."""
    pts = _f64(pts)
    P = pts.shape[0]
    nh = np.zeros(P, dtype=np.int32)
    faces = np.zeros((P, cap), dtype=np.int32)
    bary = np.zeros((P, cap, 4))
    lib().otref_query_all(_p(_f64(fwd_xy)), int(n), _p(pts), P, cap,
                          nh.ctypes.data_as(_ip), faces.ctypes.data_as(_ip), _p(bary))
    return nh, faces, bary


def rasterize(xy, n, density, rows, cols, per_vertex=False):
    """rasterize_image (otlib/utils/rasterizer.cpp:188-308); image is [y][x]."""
    img = np.zeros((rows, cols))
    d = None if density is None else _f64(density)
    sec = lib().otref_rasterize(_p(_f64(xy)), int(n), None if d is None else _p(d), int(rows),
                                int(cols), int(bool(per_vertex)), _p(img))
    return img, sec


def transport_cost(src_xy, dst_xy, n, density, per_face=False):
    """transport_cost (otlib/transport_map.cpp:131-215)."""
    pf = np.zeros(n * n) if per_face else None
    c = lib().otref_transport_cost(_p(_f64(src_xy)), _p(_f64(dst_xy)), int(n), _p(_f64(density)),
                                   None if pf is None else _p(pf))
    return (c, pf) if per_face else c


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _pi(a):
    return a.ctypes.data_as(_ip)


def rasterize_mesh(xy, start, idx, density, rows, cols, per_vertex=False):
    """rasterize_image (otlib/utils/rasterizer.cpp:188-302) of an indexed tri/quad mesh."""
    xy = _f64(xy).reshape(-1, 2)
    start, idx = _i32(start), _i32(idx)
    img = np.zeros((rows, cols))
    d = None if density is None else _f64(density)
    lib().otref_rasterize_mesh(xy.shape[0], _p(xy), start.size - 1, _pi(start), _pi(idx),
                               None if d is None else _p(d), 0 if d is None else d.size, rows, cols,
                               int(bool(per_vertex)), _p(img))
    return img


def barycenter(n, inv_meshes, alpha, beta, means, rows, cols):
    """One image of apps/barycenters.cpp:250-290 (4 maps: bilinear, 2 maps: linear).
    Returns (blended mesh, image, expected mean)."""
    ms = [_f64(m) for m in inv_meshes]
    arr = (_dp * len(ms))(*[_p(m) for m in ms])
    mv = _f64(means)
    mesh = np.empty_like(ms[0])
    img = np.zeros((rows, cols))
    e = lib().otref_barycenter(int(n), len(ms), arr, float(alpha), float(beta), _p(mv), rows, cols, _p(mesh),
                               _p(img))
    return mesh, img, e


def image_mean(img):
    """Eigen MatrixXd::mean() of an image given [y][x]."""
    img = _f64(img)
    return lib().otref_image_mean(_p(img), img.shape[0], img.shape[1])


def prune_empty_faces(xy, start, idx, density):
    """prune_empty_faces (otlib/utils/mesh_utils.cpp:124-141) on an indexed mesh."""
    xy = _f64(xy).reshape(-1, 2)
    start, idx, d = _i32(start), _i32(idx), _f64(density)
    nv, nf = C.c_int(0), C.c_int(0)
    xo = np.zeros_like(xy)
    so = np.zeros_like(start)
    io = np.zeros_like(idx)
    lib().otref_prune(xy.shape[0], _p(xy), start.size - 1, _pi(start), _pi(idx), _p(d), d.size, C.byref(nv),
                      _p(xo), C.byref(nf), _pi(so), _pi(io))
    return xo[:nv.value].copy(), so[:nf.value + 1].copy(), io[:so[nf.value]].copy()


def write_off(path, xy, start, idx):
    """Surface_mesh::write (otlib/surface_mesh/IO_off.cpp:312-380)."""
    xy = _f64(xy).reshape(-1, 2)
    start, idx = _i32(start), _i32(idx)
    ok = lib().otref_write_off(xy.shape[0], _p(xy), start.size - 1, _pi(start), _pi(idx), str(path).encode())
    if not ok:
        raise OSError(f"reference could not write {path}")


def read_off(path, cap_v, cap_f, cap_i):
    """Surface_mesh::read (otlib/surface_mesh/IO_off.cpp:255-300) -> (xy, start, idx)."""
    xy = np.zeros((cap_v, 2))
    start = np.zeros(cap_f + 1, dtype=np.int32)
    idx = np.zeros(cap_i, dtype=np.int32)
    nv, nf = C.c_int(0), C.c_int(0)
    r = lib().otref_read_off(str(path).encode(), cap_v, cap_f, cap_i, C.byref(nv), _p(xy), C.byref(nf), _pi(start),
                             _pi(idx))
    if r != 1:
        raise OSError(f"reference could not read {path} ({r})")
    return xy[:nv.value].copy(), start[:nf.value + 1].copy(), idx[:start[nf.value]].copy()


def sample_image(xy, start, idx, spf, seed, rows, cols):
    """sample_transportmap_to_image (otlib/utils/stochastic_rasterizer.cpp:19-88) after srand(seed)."""
    xy = _f64(xy).reshape(-1, 2)
    start, idx, spf = _i32(start), _i32(idx), _i32(spf)
    img = np.zeros((rows, cols))
    lib().otref_sample_image(xy.shape[0], _p(xy), start.size - 1, _pi(start), _pi(idx), _pi(spf), int(seed), rows,
                             cols, _p(img))
    return img
