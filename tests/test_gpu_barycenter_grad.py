"""The differentiable barycenter loss (otm_barycenter_loss): the barycenters demo
(apps/barycenters.cpp:184-198 inverse meshes, :250-276 blend, :280-290 raster and
rescale) as one loss L = sum (image - target)^2 and its gradient with respect to every
input density.

* forward: equal to the same pipeline composed of the public calls (batched solve,
  inverse of the origin grid, otm_barycenter);
* gradient: against an FP64 CPU chain -- the raster's area derivative with pixel
  ownership held fixed, the blend, a numerical Jacobian of the bilinear inversion
  (Newton solve, central differences) and the sparse-Jacobian adjoint reference --
  within 1e-5;
* at 512^2 with four Gaussian-mixture densities: against central differences (h = 1e-3
  .. 1e-5 relative to each density value, FP64) of the same loss with the pixel ownership
  held fixed, along the gradient's direction and smooth random directions, within 1e-3.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ot():
    from otmap_b200 import otmap

    return otmap


def tight_adjoint(tol=1e-13, restart=40, max_iter=2000):
    """Krylov adjoint to a small relative residual: the conditioning of J^T multiplies the
    solver's residual in the gradient."""
    from otmap_b200 import native as N
    import ctypes as C

    ao = N.AdjointOptionsC()
    N.lib().otm_default_adjoint_options(C.byref(ao))
    ao.mode = N.ADJOINT_KRYLOV
    ao.tol = tol
    ao.restart = restart
    ao.max_iter = max_iter
    return ao


def weights_bilinear(a, b):
    return [(1 - a) * (1 - b), a * (1 - b), a * b, (1 - a) * b]


def origin_grid(n):
    t = np.arange(n + 1, dtype=np.float64) * (1.0 / n)
    return np.stack([np.repeat(t, n + 1), np.tile(t, n + 1)], axis=1)


def signed_areas(B, n):
    P = B.reshape(n + 1, n + 1, 2)
    c = [P[:-1, :-1], P[1:, :-1], P[1:, 1:], P[:-1, 1:]]  # corners 0..3 of face (i, j)
    A = np.zeros((n, n))
    for k in range(4):
        a, b = c[k], c[(k + 1) % 4]
        A += 0.5 * (a[..., 0] * b[..., 1] - b[..., 0] * a[..., 1])
    return A.ravel(), c  # face f = j + i n  <->  [i, j]


def frozen_image(B, n, owner, expected):
    """PerFace unit-density raster of B with the given pixel ownership, rescaled to the
    expected mean (apps/barycenters.cpp:280-284); returns (image, R, s)."""
    A, _ = signed_areas(B, n)
    scale = float(np.float32(1.0 / (n * n)))
    val = scale / np.abs(A)
    R = np.where(owner >= 0, val[np.maximum(owner, 0)], 0.0)
    s = expected / R.mean()
    return R * s, R, s


def bilinear_uv(x, P, uv0):
    """Newton solve of x = (1-u)(1-v)P0 + u(1-v)P1 + uvP2 + (1-u)vP3 (vectorised)."""
    u, v = uv0[:, 0].copy(), uv0[:, 1].copy()
    for _ in range(8):
        X = ((1 - u) * (1 - v))[:, None] * P[:, 0] + (u * (1 - v))[:, None] * P[:, 1] + (u * v)[:, None] * P[:, 2] \
            + ((1 - u) * v)[:, None] * P[:, 3]
        Ju = (1 - v)[:, None] * (P[:, 1] - P[:, 0]) + v[:, None] * (P[:, 2] - P[:, 3])
        Jv = (1 - u)[:, None] * (P[:, 3] - P[:, 0]) + u[:, None] * (P[:, 2] - P[:, 1])
        r = X - x
        det = Ju[:, 0] * Jv[:, 1] - Ju[:, 1] * Jv[:, 0]
        du = (Jv[:, 1] * r[:, 0] - Jv[:, 0] * r[:, 1]) / det
        dv = (-Ju[:, 1] * r[:, 0] + Ju[:, 0] * r[:, 1]) / det
        u, v = u - du, v - dv
    return np.stack([u, v], axis=1)


def reference_chain(ot, port, n, res, dens_raw, w, target, fwds, adjs):
    """FP64 CPU gradient of the frozen-ownership loss with respect to each raw density."""
    from adjoint_ref import reference_gradient

    count = len(dens_raw)
    x = origin_grid(n)
    inv, hit0 = [], []
    for k in range(count):
        pos, _, _, _ = port.apply_inverse(fwds[k], adjs[k], n, x)
        nh, hits, _ = port.query_all(fwds[k], n, x, cap=4)
        assert (nh > 0).all()
        inv.append(pos)
        hit0.append(hits[:, 0])
    B = w[0] * inv[0]
    for k in range(1, count):
        B = B + w[k] * inv[k]
    owner = ot.raster_faces(B, res, res, n=n)
    expected = sum(w[k] * dens_raw[k].mean() for k in range(count))
    img, R, s = frozen_image(B, n, owner, expected)
    g = 2.0 * (img - target)
    sgR = (g * R).sum()
    dR = s * (g - sgR / R.sum())
    dexp = sgR / R.mean()
    A, _ = signed_areas(B, n)
    scale = float(np.float32(1.0 / (n * n)))
    dA = np.zeros(n * n)
    np.add.at(dA, owner[owner >= 0], dR[owner >= 0])
    Rf = scale / np.abs(A)
    dA = -dA * Rf / A
    # shoelace gradient back to the vertices of B
    dB = np.zeros(((n + 1), (n + 1), 2))
    P = B.reshape(n + 1, n + 1, 2)
    c = [P[:-1, :-1], P[1:, :-1], P[1:, 1:], P[:-1, 1:]]
    sl = [(slice(0, n), slice(0, n)), (slice(1, n + 1), slice(0, n)), (slice(1, n + 1), slice(1, n + 1)),
          (slice(0, n), slice(1, n + 1))]
    dA2 = dA.reshape(n, n)
    for k in range(4):
        nx, pv = c[(k + 1) % 4], c[(k + 3) % 4]
        dB[sl[k] + (0,)] += dA2 * 0.5 * (nx[..., 1] - pv[..., 1])
        dB[sl[k] + (1,)] += dA2 * 0.5 * (pv[..., 0] - nx[..., 0])
    dB = dB.reshape(-1, 2)
    grads = []
    e = 1.0 / n
    for k in range(count):
        dI = w[k] * dB
        F = fwds[k].reshape(-1, 2)
        h = hit0[k]
        i, j = h // n, h % n
        vid = np.stack([j + i * (n + 1), j + (i + 1) * (n + 1), (j + 1) + (i + 1) * (n + 1), (j + 1) + i * (n + 1)], 1)
        Pq = F[vid]  # (V, 4, 2)
        uv = bilinear_uv(x, Pq, np.full((x.shape[0], 2), 0.5))
        dF = np.zeros_like(F)

        def central(cc, d, hh):
            Pp = Pq.copy()
            Pm = Pq.copy()
            Pp[:, cc, d] += hh
            Pm[:, cc, d] -= hh
            return (bilinear_uv(x, Pp, uv) - bilinear_uv(x, Pm, uv)) / (2 * hh)

        for cc in range(4):
            for d in range(2):
                # Richardson extrapolation of central differences: the inversion is strongly
                # curved on boundary points, where a single 1e-7 step leaves ~1e-6 of error
                duv = (4.0 * central(cc, d, 1e-7) - central(cc, d, 2e-7)) / 3.0
                contrib = e * (duv * dI).sum(axis=1)  # I = O + e (u, v)
                np.add.at(dF[:, d], vid[:, cc], contrib)
        gk, _ = reference_gradient(fwds[k], dens_raw[k], dF, n)
        grads.append(gk + w[k] * dexp / (n * n))
    loss = float(((img - target) ** 2).sum())
    return loss, img, grads


def test_forward_matches_composed_pipeline(ot):
    from otmap_b200 import workloads as W

    n, res = 64, 64
    dens = [W.to_cells(W.blurred_shapes(n, 30 + k, sigma_px=1.5)) for k in range(4)]
    target = W.gaussian_mixture(res, 9)
    w = weights_bilinear(0.5, 0.5)
    loss, img, _, st = ot.barycenter_loss(dens, w, target, grad=False)
    maps = ot.solve_batch(dens)
    inv = []
    for m in maps:
        p = origin_grid(n).copy()
        m.apply_inverse(p)
        inv.append(p)
    img2, _ = ot.barycenter_image(inv, 0.5, 0.5, [d.mean() for d in dens], res)
    # the density means are summed in different orders (numpy here, a fixed tree on the GPU)
    np.testing.assert_allclose(img, img2, rtol=1e-13, atol=0)
    assert abs(loss - ((img2 - target) ** 2).sum()) <= 1e-12 * max(1.0, loss)
    assert st.inverse_missing == 0


@pytest.mark.parametrize("n,res", [(24, 24), (20, 36)])
def test_gradient_matches_fp64_reference(n, res, ot, oracle_port):
    from otmap_b200 import workloads as W

    dens = [W.to_cells(W.gaussian_mixture(n, 70 + k)) * (1.0 + 0.3 * k) for k in range(4)]
    target = W.gaussian_mixture(res, 5)
    w = weights_bilinear(0.3, 0.6)
    opt = ot.SolverOptions(threshold=0.0, max_iter=300)
    loss, img, grads, st = ot.barycenter_loss(dens, w, target, res=res, opt=opt, adjoint_opt=tight_adjoint())
    fwds, adjs = [], []
    for d in dens:
        s = ot.GridBasedTransportSolver()
        s.set_verbose_level(0)
        s.init(n)
        m = s.solve(d, opt)
        fwds.append(m.fwd_mesh())
        adjs.append(m.density())
    loss_r, img_r, grads_r = reference_chain(ot, oracle_port, n, res, dens, w, target, fwds, adjs)
    np.testing.assert_allclose(img, img_r, rtol=1e-12, atol=0)
    assert abs(loss - loss_r) <= 1e-12 * loss_r
    # 1e-5: the reference chain's numerical Jacobian of the inversion loses accuracy on
    # sliver faces (a map of the (20, 36) case has a face 1e-4 tall along the boundary,
    # where it differs from the analytic Jacobian by 1.6e-6 of the norm)
    for g, gr in zip(grads, grads_r):
        rel = np.linalg.norm(g - gr) / np.linalg.norm(gr)
        assert rel <= 1e-5, rel


def folded_corners(fwd, n):
    """Corners of the quads (v = j + i (n+1); corners (i,j), (i+1,j), (i+1,j+1), (i,j+1))
    whose turn has the opposite sign to the undeformed grid's, or none."""
    P = np.asarray(fwd).reshape(n + 1, n + 1, 2)
    q = [P[:-1, :-1], P[1:, :-1], P[1:, 1:], P[:-1, 1:]]
    G = origin_grid(n).reshape(n + 1, n + 1, 2)
    g = [G[:-1, :-1], G[1:, :-1], G[1:, 1:], G[:-1, 1:]]
    bad = 0
    for c in range(4):
        def turn(v):
            a, b, p = v[c], v[(c + 1) % 4], v[(c + 3) % 4]
            u, w_ = b - a, p - a
            return u[..., 0] * w_[..., 1] - u[..., 1] * w_[..., 0]
        bad += int((turn(q) * np.sign(turn(g)) <= 0).sum())
    return bad


def test_gradient_central_differences_512(ot):
    """Config-5 sizes (four 512^2 densities, the centre barycenter rasterized at 512^2, a
    seeded Gaussian-mixture target): directional derivatives against central differences
    of the loss with the pixel ownership of the base point held fixed, along the gradient's
    own direction and two smooth random directions, for h = 1e-3 .. 1e-5 relative to each
    density value. Gaussian-mixture densities: their forward meshes have no folded faces
    (every corner of every quad keeps the grid's orientation), so the inverse is a
    continuous function of the mesh and the loss is smooth -- an origin vertex on an edge
    shared by two faces gets the same position from either. With the sharp blurred-shape
    densities a few origin vertices fall in overlapping folded faces near the boundary,
    where the reference's inversion rule (first hit's weights, densest face) jumps, and
    finite differences pick up those jumps."""
    from otmap_b200 import workloads as W
    from otmap_b200.workloads import gaussian_blur

    n = res = 512
    # seeds whose maps are fold-free at 512^2 (seeds 60 and 62 have 448 and 866 folded
    # corners in low-density regions)
    dens = [W.to_cells(W.gaussian_mixture(n, 64 + k)) for k in range(4)]
    target = W.gaussian_mixture(res, 17)
    w = weights_bilinear(0.5, 0.5)
    # maps converged to the FP64 floor (threshold 0): a solve stopped at residual 1e-13 is
    # still ~1e-5 from its limit at this size
    opt = ot.SolverOptions(threshold=0.0, max_iter=3000)
    loss, img, grads, st = ot.barycenter_loss(dens, w, target, opt=opt,
                                              adjoint_opt=tight_adjoint(1e-12, restart=200, max_iter=8000))
    assert st.inverse_missing == 0
    assert max(st.adjoint_residual[k] for k in range(4)) <= 1e-11, list(st.adjoint_residual)[:4]

    def blend_of(ds, check_folds=False):
        maps = ot.solve_batch(ds, opt)
        B = None
        for k, m in enumerate(maps):
            if check_folds:
                assert folded_corners(m.fwd_mesh(), n) == 0
            p = origin_grid(n).copy()
            nh = np.zeros(len(p), dtype=np.int32)
            m.apply_inverse(p, None, nh)
            assert (nh >= 1).all()
            B = w[0] * p if B is None else B + w[k] * p
        return B

    blend_of(dens, check_folds=True)

    B0 = blend_of(dens)
    owner = ot.raster_faces(B0, res, res, n=n)

    def frozen_loss(ds):
        expected = sum(w[k] * ds[k].mean() for k in range(4))
        im, _, _ = frozen_image(blend_of(ds), n, owner, expected)
        return float(((im - target) ** 2).sum())

    assert abs(frozen_loss(dens) - loss) <= 1e-10 * loss
    rng = np.random.default_rng(2)
    dirs = [[g * d * d for g, d in zip(grads, dens)]]
    for _ in range(2):
        dirs.append([W.to_cells(gaussian_blur(rng.standard_normal((n, n)), 16.0)) * d for d in dens])
    for v in dirs:
        scale = max(float(np.abs(x / d).max()) for x, d in zip(v, dens))
        v = [x / scale for x in v]
        an = sum(float(g @ x) for g, x in zip(grads, v))
        for h in (1e-3, 1e-4, 1e-5):
            plus = frozen_loss([d + h * x for d, x in zip(dens, v)])
            minus = frozen_loss([d - h * x for d, x in zip(dens, v)])
            fd = (plus - minus) / (2 * h)
            assert abs(fd - an) <= 1e-3 * abs(an), (h, fd, an)
