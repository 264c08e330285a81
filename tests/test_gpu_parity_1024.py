"""Parity at the benchmarked sizes, against the reference itself (oracle/_ref: the
reference library compiled from its own sources, FP64, Eigen SimplicialLDLT).

* single large solve: a 1024^2 blurred-shape density (6 disks / convex polygons,
  sigma 5 px, floor 1e-3) to residual 1e-7 -- identical iteration count, vertex
  positions within 1e-6 of the unit square, final residual <= 1e-7
  (otsolver_2dgrid.cpp:106-245);
* its inversion: 2^20 query points drawn in FP32, located in the reference's forward
  mesh -- hit counts equal for every point, located face and inverse position
  bit-exact for every point with one containing face, and for points inside several
  faces (ties) the same face choice and position as the reference's BVH traversal
  order gives (transport_map.cpp:50-128);
* its rasterization at 1024^2 -- bit-exact (rasterizer.cpp:188-236);
* a mixed batch with one instance of every size class (128^2 .. 1024^2) at residual
  1e-6 in one batched call -- per instance the reference's iteration count and
  positions within 1e-6.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POS_TOL = 1e-6


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R

    if not R.available():
        pytest.skip("the reference library (oracle/_ref) is not built")
    return R


@pytest.fixture(scope="module")
def ot():
    from otmap_b200 import otmap

    return otmap


@pytest.fixture(scope="module")
def config2(ref, ot):
    from otmap_b200 import workloads as W

    n = 1024
    d = W.to_cells(W.blurred_shapes(n, 0, sigma_px=5.0))
    rs = ref.RefSolver()
    rs.init(n)
    rm = rs.solve(d, threshold=1e-7)
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(n)
    gm = s.solve(d, ot.SolverOptions(threshold=1e-7))
    return {"n": n, "ref_map": rm, "ref_fwd": rm.fwd(), "ref_density": rm.density(), "gpu": gm}


def test_config2_solve_1024(config2):
    rm, gm = config2["ref_map"], config2["gpu"]
    assert gm.stats.iterations == rm.iterations
    err = float(np.abs(gm.fwd_mesh() - config2["ref_fwd"]).max())
    assert err <= POS_TOL, err
    assert gm.stats.residual <= 1e-7
    # the normalisation sums 2^20 values: the reference in sequence, the GPU in a fixed tree
    np.testing.assert_allclose(gm.density(), config2["ref_density"], rtol=1e-11, atol=0)


def test_config2_inverse_2p20_points(config2, ref, ot):
    from otmap_b200 import workloads as W

    n = config2["n"]
    fwd, dens = config2["ref_fwd"], config2["ref_density"]
    pts = W.random_points(1 << 20, 7)
    # the reference: positions through apply_inverse_map, hit lists in BVH order
    pos_ref, _ = config2["ref_map"].apply_inverse(pts)
    nh_ref, faces_ref, _ = ref.query_all(fwd, n, pts)
    tm = ot.TransportMap(n, fwd, dens)
    p = np.ascontiguousarray(pts.copy())
    face = np.zeros(p.shape[0], dtype=np.int32)
    nh = np.zeros(p.shape[0], dtype=np.int32)
    missing = tm.apply_inverse(p, face, nh)
    assert missing == int((nh_ref == 0).sum()) == 0
    assert np.array_equal(nh, nh_ref)
    one = nh_ref == 1
    assert np.array_equal(face[one], faces_ref[one, 0])
    assert np.array_equal(p[one], pos_ref[one])
    ties = nh_ref > 1
    # ties: the reference keeps the first hit's weights and the densest face
    # (transport_map.cpp:70-85); the hit order is its BVH traversal order
    assert np.array_equal(p[ties], pos_ref[ties]), int((p[ties] != pos_ref[ties]).any(axis=1).sum())


def test_config2_raster_1024(config2, ref, ot):
    n = config2["n"]
    fwd, dens = config2["ref_fwd"], config2["ref_density"]
    img_ref, _ = ref.rasterize(fwd, n, dens, n, n)
    img = np.empty((n, n))
    ot.rasterize_image(fwd, dens, img, n=n)
    assert np.array_equal(img, img_ref), int((img != img_ref).sum())


def test_config3_mixed_batch_vs_reference(ref, ot):
    from otmap_b200 import workloads as W

    rng = np.random.default_rng(5)
    sizes = [128, 256, 512, 1024, 256, 128]
    imgs = [W.gaussian_mixture(n, 600 + k, k=int(rng.integers(4, 17))) for k, n in enumerate(sizes)]
    opt = ot.SolverOptions(threshold=1e-6)
    maps = ot.solve_batch(imgs, opt)
    solvers = {}
    for img, m in zip(imgs, maps):
        n = img.shape[0]
        if n not in solvers:
            solvers[n] = ref.RefSolver()
            solvers[n].init(n)
        r = solvers[n].solve(W.to_cells(img), threshold=1e-6)
        assert m.stats.iterations == r.iterations, (n, m.stats.iterations, r.iterations)
        err = float(np.abs(m.fwd_mesh() - r.fwd()).max())
        assert err <= POS_TOL, (n, err)
        assert m.stats.residual <= 1e-6
