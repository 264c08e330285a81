"""Seeded synthetic densities for the solver's benchmark and parity workloads.

No public dataset is involved: every workload is generated here on the host in
FP64, deterministically from a seed, and the same bytes are fed to the GPU solver
and to the CPU reference.

Layout: generators return images ``img[y, x]`` of shape (n, n). The solver's
per-cell buffers use the reference's face index ``f = j + i*n`` with ``i`` the x
cell index and ``j`` the y cell index (otlib/otsolver_2dgrid.h:90), i.e. the
column-major flattening of the image (apps/common/generic_tasks.cpp:67 passes
``vec(MatrixXd)``); :func:`to_cells` and :func:`from_cells` convert.

Workloads (sizes from the solver's published configurations):
  * :func:`gaussian_mixture` -- 8 isotropic Gaussians (centres U[0.1,0.9]^2,
    sigma U[0.03,0.15], amplitude U[0.5,2]) + floor 1e-3, mean 1. 256^2 plain run.
  * :func:`blurred_shapes` -- 6 filled disks / convex polygons (value 1,
    background 1e-3), Gaussian blur sigma=5 px, mean 1. 1024^2 single solve.
  * :func:`batched_mixtures` -- 64 instances, n log-uniform over
    {128,256,512,1024}, 4..16 Gaussians each, floor 1e-3.
  * :func:`softmax_logits` -- softmax of N(0,1) logits, blur sigma=8 px (512^2).
"""

from __future__ import annotations

import math

import numpy as np

__all__ = [
    "to_cells",
    "from_cells",
    "gaussian_mixture",
    "blurred_shapes",
    "batched_mixtures",
    "softmax_logits",
    "gaussian_blur",
    "random_points",
]


def to_cells(img: np.ndarray) -> np.ndarray:
    """Image ``img[y, x]`` -> per-cell vector in face order ``f = y + x*n``."""
    img = np.asarray(img, dtype=np.float64)
    return np.ascontiguousarray(img.ravel(order="F"))


def from_cells(vec: np.ndarray, n: int) -> np.ndarray:
    """Per-cell vector in face order -> image ``img[y, x]``."""
    return np.asarray(vec, dtype=np.float64).reshape(n, n).T.copy()


def _cell_centres(n: int):
    c = (np.arange(n, dtype=np.float64) + 0.5) / n
    x = c[None, :]  # columns are x
    y = c[:, None]  # rows are y
    return x, y


def _normalise(img: np.ndarray) -> np.ndarray:
    return img / img.mean()


def gaussian_mixture(n: int, seed: int, k: int = 8, floor: float = 1e-3) -> np.ndarray:
    """Sum of ``k`` isotropic Gaussians plus ``floor``, normalised to mean 1."""
    rng = np.random.default_rng(seed)
    x, y = _cell_centres(n)
    img = np.zeros((n, n), dtype=np.float64)
    for _ in range(k):
        cx, cy = rng.uniform(0.1, 0.9, size=2)
        s = rng.uniform(0.03, 0.15)
        a = rng.uniform(0.5, 2.0)
        img += a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * s * s))
    return _normalise(img + floor)


def _gauss_kernel(sigma: float) -> np.ndarray:
    r = max(1, int(math.ceil(3.0 * sigma)))
    t = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (t / sigma) ** 2)
    return k / k.sum()


def gaussian_blur(img: np.ndarray, sigma: float) -> np.ndarray:
    """Separable Gaussian blur (radius ceil(3 sigma), mirror borders), FP64."""
    if sigma <= 0:
        return np.array(img, dtype=np.float64)
    k = _gauss_kernel(sigma)
    r = (len(k) - 1) // 2
    out = np.asarray(img, dtype=np.float64)
    for axis in (0, 1):
        pad = [(0, 0), (0, 0)]
        pad[axis] = (r, r)
        p = np.pad(out, pad, mode="symmetric")
        acc = np.zeros_like(out)
        for t in range(len(k)):
            sl = [slice(None), slice(None)]
            sl[axis] = slice(t, t + out.shape[axis])
            acc += k[t] * p[tuple(sl)]
        out = acc
    return out


def blurred_shapes(n: int, seed: int, count: int = 6, sigma_px: float = 5.0,
                   background: float = 1e-3) -> np.ndarray:
    """``count`` filled disks or convex polygons (value 1) on ``background``,
    Gaussian-blurred with ``sigma_px`` pixels, normalised to mean 1."""
    rng = np.random.default_rng(seed)
    x, y = _cell_centres(n)
    img = np.full((n, n), background, dtype=np.float64)
    for _ in range(count):
        cx, cy = rng.uniform(0.2, 0.8, size=2)
        rad = rng.uniform(0.05, 0.15)
        if rng.uniform() < 0.5:
            inside = (x - cx) ** 2 + (y - cy) ** 2 <= rad * rad
        else:
            m = int(rng.integers(3, 9))
            ang = np.sort(rng.uniform(0.0, 2.0 * math.pi, size=m))
            px = cx + rad * np.cos(ang)
            py = cy + rad * np.sin(ang)
            inside = np.ones((n, n), dtype=bool)
            # vertices sorted by angle form a convex polygon, counter-clockwise
            for q in range(m):
                ax, ay = px[q], py[q]
                bx, by = px[(q + 1) % m], py[(q + 1) % m]
                inside &= (bx - ax) * (y - ay) - (by - ay) * (x - ax) >= 0.0
        img[inside] = 1.0
    return _normalise(gaussian_blur(img, sigma_px))


def batched_mixtures(count: int = 64, seed: int = 0,
                     sizes=(128, 256, 512, 1024), floor: float = 1e-3):
    """``count`` Gaussian mixtures (4..16 components) with n drawn uniformly over
    ``sizes`` (log-uniform in n). Returns a list of images."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(sizes[int(rng.integers(0, len(sizes)))])
        k = int(rng.integers(4, 17))
        out.append(gaussian_mixture(n, int(rng.integers(0, 2**31 - 1)), k=k, floor=floor))
    return out


def softmax_logits(n: int, seed: int, sigma_px: float = 8.0):
    """Logits z ~ N(0,1) per cell, density = blur(softmax(z)) normalised to mean 1.
    Returns (logits image, density image)."""
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((n, n))
    e = np.exp(z - z.max())
    p = e / e.sum()
    return z, _normalise(gaussian_blur(p, sigma_px))


def random_points(count: int, seed: int) -> np.ndarray:
    """``count`` points uniform in [0,1]^2 drawn in FP32, returned as FP64 (count, 2)."""
    rng = np.random.default_rng(seed)
    return rng.random((count, 2), dtype=np.float32).astype(np.float64)
