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

    def release(self):
        """Frees the device map (the point locator); it is rebuilt on the next inverse."""
        m = getattr(self, "_map", None)
        self._map = None
        if m is not None:
            _n.lib().otm_map_destroy(m)

    def __del__(self):
        try:
            self.release()
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
            self._ctx.track(self)
        return self._map

    def init_inverse(self):
        """transport_map.cpp:36-43"""
        _n.check(_n.lib().otm_map_init_inverse(self._device_map()))

    def inv(self, p) -> np.ndarray:
        """transport_map.h:44 for one point."""
        q = np.array(p, dtype=np.float64).reshape(1, 2)
        self.apply_inverse(q)
        return q[0]

    def inv_fast(self, p) -> np.ndarray:
        """transport_map.h:45: the first containing face (lowest index) and its weights."""
        q = np.array(p, dtype=np.float64).reshape(1, 2)
        self.apply_inverse(q, fast=True)
        return q[0]

    def apply_inverse(self, points, face=None, nhits=None, fast: bool = False) -> int:
        """In place on a (P, 2) float64 array -- a numpy array or a CUDA tensor, which then
        stays on the device; returns the number of points with no face. fast=False chooses
        faces as inv does, fast=True as inv_fast."""
        import ctypes as C

        if hasattr(points, "data_ptr"):
            import torch

            if points.dtype != torch.float64 or not points.is_contiguous() or points.dim() != 2 or points.shape[1] != 2:
                raise TypeError("points must be a contiguous float64 (P, 2) tensor")
        elif points.dtype != np.float64 or not points.flags["C_CONTIGUOUS"]:
            raise TypeError("points must be a C-contiguous float64 (P, 2) array")
        missing = C.c_long(0)
        mode = _n.INV_FIRST if fast else _n.INV_DENSEST
        _n.check(_n.lib().otm_map_inverse_mode(self._device_map(), _n.ptr(points), points.shape[0], mode,
                                               _n.ptr(face), _n.ptr(nhits), C.byref(missing)))
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


class RasterImageOption(enum.IntEnum):
    """otmap::RasterImageOption (utils/rasterizer.h:16-19)."""

    RIO_PerVertexDensity = 0
    RIO_PerFaceDensity = 1


RIO_PerVertexDensity = RasterImageOption.RIO_PerVertexDensity
RIO_PerFaceDensity = RasterImageOption.RIO_PerFaceDensity


@dataclass
class Mesh:
    """A triangle/quad mesh as an indexed face set: vertex positions (V, 2) and face f's
    corners face_vertices[face_start[f]:face_start[f+1]] in circulation order. The
    counterpart of the reference's Surface_mesh for meshes other than the grid."""

    xy: np.ndarray
    face_start: np.ndarray
    face_vertices: np.ndarray

    @staticmethod
    def grid(n: int, xy: np.ndarray | None = None) -> "Mesh":
        """The (n+1)^2 grid mesh (mesh_utils.cpp:90-122), at `xy` (default: the origin grid)."""
        start = np.empty(n * n + 1, dtype=np.int32)
        idx = np.empty(4 * n * n, dtype=np.int32)
        _n.check(_n.lib().otm_grid_faces(n, _n.ptr(start), _n.ptr(idx)))
        pts = grid_vertices(n) if xy is None else np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
        return Mesh(pts.copy(), start, idx)

    @property
    def n_vertices(self) -> int:
        return int(self.xy.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.face_start.size - 1)

    def _arrays(self):
        return (np.ascontiguousarray(self.xy, dtype=np.float64).reshape(-1, 2),
                np.ascontiguousarray(self.face_start, np.int32), np.ascontiguousarray(self.face_vertices, np.int32))

    def write(self, path: str) -> None:
        """Surface_mesh::write for .off (surface_mesh/IO_off.cpp:312-380)."""
        xy, st, ix = self._arrays()
        _n.check(_n.lib().otm_write_off(str(path).encode(), xy.shape[0], _n.ptr(xy), st.size - 1, _n.ptr(st),
                                        _n.ptr(ix)))

    @staticmethod
    def read(path: str) -> "Mesh":
        """Surface_mesh::read for .off (surface_mesh/IO_off.cpp:45-300)."""
        import ctypes as C

        nv, nf, ni = C.c_int(0), C.c_int(0), C.c_int(0)
        _n.check(_n.lib().otm_read_off(str(path).encode(), C.byref(nv), C.byref(nf), C.byref(ni), None, None, None))
        xy = np.empty((nv.value, 2))
        st = np.empty(nf.value + 1, dtype=np.int32)
        ix = np.empty(max(ni.value, 1), dtype=np.int32)
        _n.check(_n.lib().otm_read_off(str(path).encode(), C.byref(nv), C.byref(nf), C.byref(ni), _n.ptr(xy),
                                       _n.ptr(st), _n.ptr(ix)))
        return Mesh(xy, st, ix[:ni.value].copy())


def _grid_n(xy: np.ndarray, n: int | None) -> int:
    if n is None:
        n = int(round(np.sqrt(xy.shape[0]))) - 1
    if n < 1 or (n + 1) ** 2 != xy.shape[0]:
        raise ValueError("mesh is not an (n+1)^2 grid")
    return n


def write_off(path: str, mesh, n: int | None = None) -> None:
    """Writes a grid mesh ((V, 2) vertex array) or a Mesh as .off, as Surface_mesh::write."""
    if not isinstance(mesh, Mesh):
        xy = np.ascontiguousarray(mesh, dtype=np.float64).reshape(-1, 2)
        mesh = Mesh.grid(_grid_n(xy, n), xy)
    mesh.write(path)


def rasterize_image(mesh, density_per_face, img: np.ndarray, opt: RasterImageOption = RIO_PerFaceDensity,
                    n: int | None = None, context=None) -> None:
    """rasterize_image (rasterizer.cpp:188-308) into the pre-sized float64 array
    img[rows, cols] (row = y). mesh is the (V, 2) vertex array of an (n+1)^2 grid mesh
    or a Mesh of triangles and quads; density_per_face None = unit density."""
    ctx = context or _n.default_context()
    if img.dtype != np.float64 or not img.flags["C_CONTIGUOUS"]:
        raise TypeError("img must be a C-contiguous float64 array")
    rows, cols = img.shape
    opt = int(opt)
    if isinstance(mesh, Mesh):
        xy, st, ix = mesh._arrays()
        d = None if density_per_face is None else np.ascontiguousarray(density_per_face, dtype=np.float64).ravel()
        _n.check(_n.lib().otm_rasterize_mesh(ctx.handle, xy.shape[0], _n.ptr(xy), st.size - 1, _n.ptr(st),
                                             _n.ptr(ix), _n.ptr(d), 0 if d is None else d.size, rows, cols, opt,
                                             _n.ptr(img)))
        return
    xy = np.ascontiguousarray(mesh, dtype=np.float64).reshape(-1, 2)
    n = _grid_n(xy, n)
    d = None if density_per_face is None else _as_cells(density_per_face)
    _n.check(_n.lib().otm_rasterize_mode(ctx.handle, n, _n.ptr(xy), _n.ptr(d), rows, cols, opt, _n.ptr(img)))


def transport_cost(src_mesh, dst_mesh, density_per_face, cost_per_face: bool = False, context=None):
    """transport_cost (transport_map.h:70, transport_map.cpp:131-215) between two
    (n+1)^2 grid meshes; with cost_per_face=True returns (cost, per-face costs)."""
    import ctypes as C

    ctx = context or _n.default_context()
    src = np.ascontiguousarray(src_mesh, dtype=np.float64).reshape(-1, 2)
    dst = np.ascontiguousarray(dst_mesh, dtype=np.float64).reshape(-1, 2)
    n = _grid_n(src, None)
    if dst.shape != src.shape:
        raise ValueError("meshes differ in size")
    d = _as_cells(density_per_face)
    if d.size != n * n:
        raise ValueError("density does not match the mesh")
    pf = np.empty(n * n) if cost_per_face else None
    c = C.c_double(0)
    _n.check(_n.lib().otm_transport_cost(ctx.handle, n, _n.ptr(src), _n.ptr(dst), _n.ptr(d), _n.ptr(pf), C.byref(c)))
    return (c.value, pf) if cost_per_face else c.value


def grid_transport_cost(vertex_displacements, density, per_face: bool = False, context=None):
    """GridBasedTransportSolver::compute_transport_cost (otsolver_2dgrid.cpp:608-640):
    the solver's Gauss-quadrature cost of the (V, 2) vertex displacements (a map's
    fwd_mesh() - origin_mesh()); returns the sum, or (sum, per-face costs)."""
    import ctypes as C

    ctx = context or _n.default_context()
    g = np.ascontiguousarray(vertex_displacements, dtype=np.float64).reshape(-1, 2)
    n = _grid_n(g, None)
    d = _as_cells(density)
    pf = np.empty(n * n) if per_face else None
    t = C.c_double(0)
    _n.check(_n.lib().otm_grid_transport_cost(ctx.handle, n, _n.ptr(g), _n.ptr(d), _n.ptr(pf), C.byref(t)))
    return (t.value, pf) if per_face else t.value


def prune_empty_faces(mesh, density) -> Mesh:
    """prune_empty_faces (mesh_utils.cpp:124-141) on a grid vertex array or a Mesh;
    returns the pruned Mesh (the reference edits its Surface_mesh in place)."""
    import ctypes as C

    if not isinstance(mesh, Mesh):
        xy = np.ascontiguousarray(mesh, dtype=np.float64).reshape(-1, 2)
        mesh = Mesh.grid(_grid_n(xy, None), xy)
    xy, st, ix = mesh._arrays()
    d = np.ascontiguousarray(density, dtype=np.float64).ravel()
    xo = np.empty_like(xy)
    so = np.empty_like(st)
    io = np.empty_like(ix)
    nv, nf = C.c_int(0), C.c_int(0)
    _n.check(_n.lib().otm_prune_empty_faces(xy.shape[0], _n.ptr(xy), st.size - 1, _n.ptr(st), _n.ptr(ix), _n.ptr(d),
                                            d.size, C.byref(nv), _n.ptr(xo), C.byref(nf), _n.ptr(so), _n.ptr(io)))
    return Mesh(xo[:nv.value].copy(), so[:nf.value + 1].copy(), io[:so[nf.value]].copy())


def sample_transportmap_to_image(mesh, samples_per_face, img: np.ndarray, seed: int = 0, context=None) -> None:
    """sample_transportmap_to_image (stochastic_rasterizer.cpp:19-88) into the pre-sized
    float64 img[rows, cols]: samples_per_face[f] random points per face (an int, or one
    per face), counted per pixel. Reproducible from `seed` (a counter-based generator
    in place of the reference's std::rand())."""
    ctx = context or _n.default_context()
    if img.dtype != np.float64 or not img.flags["C_CONTIGUOUS"]:
        raise TypeError("img must be a C-contiguous float64 array")
    rows, cols = img.shape
    if isinstance(mesh, Mesh):
        xy, st, ix = mesh._arrays()
        grid_n, nf = 0, st.size - 1
    else:
        xy = np.ascontiguousarray(mesh, dtype=np.float64).reshape(-1, 2)
        grid_n = _grid_n(xy, None)
        nf, st, ix = grid_n * grid_n, None, None
    spf = np.broadcast_to(np.asarray(samples_per_face, dtype=np.int32), (nf,))
    spf = np.ascontiguousarray(spf)
    _n.check(_n.lib().otm_sample_image(ctx.handle, xy.shape[0], _n.ptr(xy), nf, _n.ptr(st), _n.ptr(ix), grid_n,
                                       _n.ptr(spf), int(seed) & 0xFFFFFFFFFFFFFFFF, rows, cols, _n.ptr(img)))


def synthetize_image(map_mesh, img_res: int, target, input_density=None, samples_per_face: int = 300,
                     seed: int = 0, context=None):
    """The two renderings of a map in apps/common/generic_tasks.cpp:71-99: stochastic
    samples (samples per face proportional to input_density, or constant) scaled to the
    target's mass, and the unit-density raster scaled to the target's mean. Returns
    (sampled image, raster image), both img_res x img_res, row = y."""
    t = np.asarray(target, dtype=np.float64).ravel()
    if isinstance(map_mesh, Mesh):
        nf = map_mesh.n_faces
    else:
        nf = _grid_n(np.asarray(map_mesh).reshape(-1, 2), None) ** 2
    if input_density is not None:
        d = np.asarray(input_density, dtype=np.float64).ravel()
        spf = (samples_per_face * d.size / d.sum() * d).astype(np.int32)
        if nf == 2 * spf.size:  # a grid of triangles: two faces per cell
            spf = np.repeat(spf, 2)
    else:
        spf = np.full(nf, samples_per_face, dtype=np.int32)
    sampled = np.empty((img_res, img_res))
    sample_transportmap_to_image(map_mesh, spf, sampled, seed, context)
    sampled *= t.sum() / float(samples_per_face * nf)
    raster = np.empty((img_res, img_res))
    rasterize_image(map_mesh, None, raster, context=context)
    raster = raster * t.sum() / t.size
    return sampled, raster


def bilinear_weights(alpha: float, beta: float):
    """Weights of bilerp(alpha, beta, a0..a3) (apps/barycenters.cpp:127-134)."""
    a, b = float(alpha), float(beta)
    return [(1. - a) * (1. - b), a * (1. - b), a * b, (1. - a) * b]


def linear_weights(alpha: float):
    """Weights of lerp(alpha, a0, a1) (apps/barycenters.cpp:136-139)."""
    a = float(alpha)
    return [1. - a, a]


def _as_mesh(m):
    """(V, 2) float64 vertex array: a CUDA tensor is passed through (device pointer)."""
    if hasattr(m, "data_ptr"):
        return m.reshape(-1, 2).contiguous()
    return np.ascontiguousarray(m, dtype=np.float64).reshape(-1, 2)


def _blend_args(inv_maps, alpha, beta):
    ms = [_as_mesh(m) for m in inv_maps]
    if len(ms) == 4 and beta is not None:
        w = bilinear_weights(alpha, beta)
    elif len(ms) == 2:
        w = linear_weights(alpha)
    else:
        raise ValueError("barycenters take 2 maps (alpha) or 4 maps (alpha, beta)")
    return ms, w


def interpolate(inv_maps, alpha: float, beta: float | None = None, context=None) -> np.ndarray:
    """interpolate (apps/barycenters.cpp:250-276): the bilinear (4 maps, alpha and beta)
    or linear (2 maps) blend of inverse meshes, vertex by vertex, on the GPU."""
    import ctypes as C

    ctx = context or _n.default_context()
    ms, w = _blend_args(inv_maps, alpha, beta)
    n = _grid_n(ms[0], None)
    out = np.empty((ms[0].shape[0], 2))
    arr = (C.c_void_p * len(ms))(*[_n.ptr(m).value for m in ms])
    wc = (C.c_double * len(w))(*w)
    _n.check(_n.lib().otm_mesh_blend(ctx.handle, n, len(ms), arr, wc, _n.ptr(out)))
    return out


def barycenter_image(inv_maps, alpha: float, beta: float | None, density_means, res: int, context=None,
                     want_mesh: bool = True):
    """One image of the barycenters demo (apps/barycenters.cpp:250-290): interpolate the
    inverse meshes (numpy arrays, or CUDA tensors that stay on the device), rasterize with
    unit density at res x res, rescale to the blended mean of the input densities. Returns
    (image[res, res], blended mesh, or None when want_mesh is False)."""
    import ctypes as C

    ctx = context or _n.default_context()
    ms, w = _blend_args(inv_maps, alpha, beta)
    m = [float(x) for x in density_means]
    if len(ms) == 4:
        a, b = float(alpha), float(beta)
        expected = (1. - a) * (1. - b) * m[0] + a * (1. - b) * m[1] + a * b * m[2] + (1. - a) * b * m[3]
    else:
        a = float(alpha)
        expected = (1. - a) * m[0] + a * m[1]
    n = _grid_n(ms[0], None)
    img = np.empty((res, res))
    mesh = np.empty((ms[0].shape[0], 2)) if want_mesh else None
    arr = (C.c_void_p * len(ms))(*[_n.ptr(x).value for x in ms])
    wc = (C.c_double * len(w))(*w)
    _n.check(_n.lib().otm_barycenter(ctx.handle, n, len(ms), arr, wc, expected, res, res, _n.ptr(mesh), _n.ptr(img),
                                     None))
    return img, mesh


def raster_faces(mesh: np.ndarray, rows: int, cols: int, n: int | None = None, context=None) -> np.ndarray:
    """The face index each pixel of the PerFace raster of a grid mesh takes its value from
    ([rows, cols] int32, -1 where no face covers the pixel centre)."""
    ctx = context or _n.default_context()
    xy = np.ascontiguousarray(mesh, dtype=np.float64).reshape(-1, 2)
    n = _grid_n(xy, n)
    out = np.empty((rows, cols), dtype=np.int32)
    _n.check(_n.lib().otm_rasterize_faces(ctx.handle, n, _n.ptr(xy), rows, cols, _n.ptr(out)))
    return out


def barycenter_loss(densities, weights, target, res: int | None = None, opt: SolverOptions | None = None,
                    adjoint_opt=None, grad: bool = True, context=None):
    """The barycenters demo (apps/barycenters.cpp:184-198, 250-290) as one differentiable
    loss: maps of `densities` (up to 8 per-cell vectors or square images of one size n) in
    one batch, inverse meshes of the origin grid, the blend with `weights`, its raster at
    res x res rescaled to the blended density mean, and L = sum (image - target)^2.
    Returns (loss, image[res, res], grads (list of per-cell gradients, or None), stats)."""
    import ctypes as C

    ctx = context or _n.default_context()
    cells = [_as_cells(d) for d in densities]
    count = len(cells)
    n = int(round(np.sqrt(cells[0].size)))
    t = np.ascontiguousarray(target, dtype=np.float64)
    res = int(res or t.shape[0])
    if t.shape != (res, res):
        raise ValueError("target must be res x res")
    w = (C.c_double * count)(*[float(x) for x in weights])
    dp = (C.c_void_p * count)(*[c.ctypes.data for c in cells])
    img = np.empty((res, res))
    loss = C.c_double(0.0)
    grads = [np.empty(n * n) for _ in range(count)] if grad else None
    gp = (C.c_void_p * count)(*[g.ctypes.data for g in grads]) if grad else None
    st = _n.BarycenterStatsC()
    o = (opt or SolverOptions()).to_c()
    _n.check(_n.lib().otm_barycenter_loss(ctx.handle, n, count, dp, w, res, _n.ptr(t), C.byref(o),
                                          C.byref(adjoint_opt) if adjoint_opt is not None else None, _n.ptr(img),
                                          C.byref(loss), gp, C.byref(st)))
    return loss.value, img, grads, st


def compose(tmap_u: TransportMap, tmap_v: TransportMap, verbose_level: int = 0) -> np.ndarray:
    """The map u -> v of apps/otmap.cpp:120-126: map u's forward mesh pulled through the
    inverse of map v. Returns the composite (n_u+1)^2 vertex array."""
    pts = np.array(tmap_u.fwd_mesh(), dtype=np.float64, copy=True)
    apply_inverse_map(tmap_v, pts, verbose_level)
    return pts


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
