"""Python mirror of the reference's public API (namespace otmap of ggael/otmap,
otlib/otsolver_2dgrid.h, otlib/transport_map.h, otlib/utils/rasterizer.h), running
on the GPU through the C ABI (include/otmap_b200.h). Same names, argument meaning
and behaviour: solve() always returns a map, converged or not; diagnostics go to
stdout at the verbose level the caller sets.

Buffers follow the reference's memory layouts: densities are per-cell vectors in
face order f = j + i*n (x index i, y index j; a column-major image flattened),
meshes are (V, 2) arrays of vertex positions in vertex order v = j + i*(n+1).
"""

from __future__ import annotations

import enum
import sys
from dataclasses import dataclass

import numpy as np

from . import native as _n

DBL_MAX = float(np.finfo(np.float64).max)


class BetaOpt(enum.IntEnum):
    """otmap::BetaOpt (otsolver_2dgrid.h:33-35)."""

    Zero = 0
    ConjugateJacobian = 1


@dataclass
class SolverOptions:
    """otmap::SolverOptions (otsolver_2dgrid.h:37-43)."""

    beta: BetaOpt = BetaOpt.ConjugateJacobian
    max_iter: int = 1000
    threshold: float = 1e-7
    max_ratio: float = DBL_MAX

    def to_c(self):
        o = _n.SolverOptionsC()
        o.beta = int(self.beta)
        o.max_iter = int(self.max_iter)
        o.threshold = float(self.threshold)
        o.max_ratio = float(self.max_ratio)
        return o


def grid_vertices(n: int) -> np.ndarray:
    """Regular (n+1)^2 grid, vertex v = j + i*(n+1) at (i/n, j/n) (mesh_utils.cpp:90-122)."""
    t = np.arange(n + 1, dtype=np.float64) * (1.0 / n)
    return np.stack([np.repeat(t, n + 1), np.tile(t, n + 1)], axis=1)


def _as_cells(density, n=None) -> np.ndarray:
    d = np.asarray(density, dtype=np.float64)
    if d.ndim == 2:
        if d.shape[0] != d.shape[1]:
            raise ValueError("density image must be square")
        d = d.ravel(order="F")
    return np.ascontiguousarray(d)


class TransportMap:
    """otmap::TransportMap (transport_map.h:29-63): origin grid, forward mesh and the
    adjusted density; the inverse is located on the GPU (built lazily)."""

    def __init__(self, n: int, fwd_mesh: np.ndarray, density: np.ndarray, context=None, stats=None):
        self.n = int(n)
        self._fwd = np.ascontiguousarray(fwd_mesh, dtype=np.float64).reshape(-1, 2)
        self._density = np.ascontiguousarray(density, dtype=np.float64).ravel()
        self._ctx = context or _n.default_context()
        self._map = None
        self.stats = stats

    def __del__(self):
        m = getattr(self, "_map", None)
        if m is not None:
            try:
                _n.lib().otm_map_destroy(m)
            except Exception:
                pass

    def origin_mesh(self) -> np.ndarray:
        return grid_vertices(self.n)

    def fwd_mesh(self) -> np.ndarray:
        return self._fwd

    def density(self) -> np.ndarray:
        return self._density

    def _device_map(self):
        if self._map is None:
            import ctypes as C

            h = C.c_void_p()
            _n.check(_n.lib().otm_map_create(self._ctx.handle, self.n, _n.ptr(self._fwd), _n.ptr(self._density),
                                             C.byref(h)))
            self._map = h
        return self._map

    def init_inverse(self):
        """transport_map.cpp:36-43"""
        _n.check(_n.lib().otm_map_init_inverse(self._device_map()))

    def inv(self, p) -> np.ndarray:
        """transport_map.h:44 for one point."""
        q = np.array(p, dtype=np.float64).reshape(1, 2)
        self.apply_inverse(q)
        return q[0]

    def apply_inverse(self, points: np.ndarray, face=None, nhits=None) -> int:
        """In place on a (P, 2) float64 array; returns the number of points with no face."""
        import ctypes as C

        if points.dtype != np.float64 or not points.flags["C_CONTIGUOUS"]:
            raise TypeError("points must be a C-contiguous float64 (P, 2) array")
        missing = C.c_long(0)
        _n.check(_n.lib().otm_map_inverse(self._device_map(), _n.ptr(points), points.shape[0], _n.ptr(face),
                                          _n.ptr(nhits), C.byref(missing)))
        return missing.value


class GridBasedTransportSolver:
    """otmap::GridBasedTransportSolver (otsolver_2dgrid.h:45-125)."""

    def __init__(self, context=None):
        self._ctx = context or _n.default_context()
        self._verbose = 1
        self._n = None
        self.last_stats = None

    def set_verbose_level(self, v: int):
        self._verbose = int(v)

    def init(self, n: int):
        """otsolver_2dgrid.cpp:75-104"""
        if self._n == n:
            return
        if self._verbose >= 1:
            print("Init solver...")
        self._ctx.init(n)
        self._n = int(n)

    def solve(self, density, opt: SolverOptions | None = None) -> TransportMap:
        """otsolver_2dgrid.cpp:106-245"""
        import ctypes as C

        opt = opt or SolverOptions()
        if self._n is None:
            raise RuntimeError("init(n) must be called before solve()")
        n = self._n
        d = _as_cells(density)
        if d.size != n * n:
            raise ValueError(f"density has {d.size} cells, expected {n * n}")
        fwd = np.empty(((n + 1) ** 2, 2))
        adj = np.empty(n * n)
        st = _n.SolveStatsC()
        if self._verbose >= 1:
            b = "0" if opt.beta == BetaOpt.Zero else "Conjugate-Jacobian"
            print(f" Solve transport map using beta={b} ;  max_iter={opt.max_iter} ;  threshold={opt.threshold}",
                  end="")
        c = opt.to_c()
        _n.check(_n.lib().otm_solve(self._ctx.handle, n, _n.ptr(d), C.byref(c), _n.ptr(fwd), _n.ptr(adj),
                                    C.byref(st)))
        self.last_stats = st
        if self._verbose >= 1:
            print(f"  ; initial L2={st.initial_residual}")
            print(f" Solution:\n  - iters({st.iterations})\n  - error L2={st.residual}   Linf={st.linf}")
        return TransportMap(n, fwd, adj, self._ctx, stats=st)


def apply_inverse_map(tmap: TransportMap, points: np.ndarray, verbose_level: int = 2) -> None:
    """apply_inverse_map (transport_map.cpp:105-128), in place on a (P, 2) array."""
    tmap.init_inverse()
    missing = tmap.apply_inverse(points)
    if missing and verbose_level >= 1:
        print(f"Error: no face found for {missing} point(s).", file=sys.stderr)


def rasterize_image(mesh: np.ndarray, density_per_face, img: np.ndarray, n: int | None = None,
                    context=None) -> None:
    """rasterize_image (rasterizer.cpp:188-308), PerFace mode, into the pre-sized
    float64 array img[rows, cols] (row = y). mesh is the (V, 2) vertex array of an
    (n+1)^2 grid mesh; density_per_face None = unit density."""
    ctx = context or _n.default_context()
    mesh = np.ascontiguousarray(mesh, dtype=np.float64)
    if n is None:
        n = int(round(np.sqrt(mesh.shape[0]))) - 1
    if (n + 1) ** 2 != mesh.shape[0]:
        raise ValueError("mesh is not an (n+1)^2 grid")
    if img.dtype != np.float64 or not img.flags["C_CONTIGUOUS"]:
        raise TypeError("img must be a C-contiguous float64 array")
    d = None if density_per_face is None else _as_cells(density_per_face)
    rows, cols = img.shape
    _n.check(_n.lib().otm_rasterize(ctx.handle, n, _n.ptr(mesh), _n.ptr(d), rows, cols, _n.ptr(img)))


def solve_batch(densities, opt: SolverOptions | None = None, context=None):
    """Many independent solves (uneven sizes allowed) in one GPU run; returns maps."""
    import ctypes as C

    ctx = context or _n.default_context()
    opt = opt or SolverOptions()
    cells = [_as_cells(d) for d in densities]
    ns = [int(round(np.sqrt(c.size))) for c in cells]
    fwds = [np.empty(((n + 1) ** 2, 2)) for n in ns]
    adjs = [np.empty(n * n) for n in ns]
    cnt = len(cells)
    stats = (_n.SolveStatsC * cnt)()
    ns_c = (C.c_int * cnt)(*ns)
    dp = (C.c_void_p * cnt)(*[c.ctypes.data for c in cells])
    fp = (C.c_void_p * cnt)(*[f.ctypes.data for f in fwds])
    ap = (C.c_void_p * cnt)(*[a.ctypes.data for a in adjs])
    c = opt.to_c()
    _n.check(_n.lib().otm_solve_batch(ctx.handle, cnt, ns_c, dp, C.byref(c), fp, ap, stats))
    return [TransportMap(n, f, a, ctx, stats=stats[k]) for k, (n, f, a) in enumerate(zip(ns, fwds, adjs))]
