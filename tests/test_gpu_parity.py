"""Parity of the CUDA path (through the C ABI) with the reference's golden vectors
and the C oracle. Tolerances: vertex positions within 1e-6 of the unit square (the
FP64 solver), identical iteration counts; point location and rasterization
bit-exact."""

import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

POS_TOL = 1e-6


def chosen_faces(hits, nhits, density):
    """The face inv_impl keeps (transport_map.cpp:70-85): the first hit, replaced by a
    later hit whose density exceeds `best_area`, which holds the first hit's density and,
    after a replacement, the comparison's bool. Hits are in the reference's BVH order."""
    out = np.full(len(nhits), -1, dtype=np.int64)
    for i, nh in enumerate(nhits):
        if nh == 0:
            continue
        f = hits[i, 0]
        best = density[f]
        for k in range(1, min(nh, hits.shape[1])):
            if density[hits[i, k]] > best:
                f = hits[i, k]
                best = float(density[hits[i, k]] > best)
        out[i] = f
    return out


@pytest.fixture(scope="module")
def ot():
    from otmap_b200 import otmap

    return otmap


def _solve(ot, g):
    n = int(g["n"])
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(n)
    opt = ot.SolverOptions(beta=ot.BetaOpt(int(g["beta_cj"])), max_iter=int(g["max_iter"]),
                           threshold=float(g["threshold"]), max_ratio=float(g["max_ratio"]))
    return s.solve(g["density"], opt)


@pytest.mark.parametrize("name", golden_names("solve_"))
def test_solve_matches_reference(name, ot):
    g = load_golden(name)
    m = _solve(ot, g)
    assert m.stats.iterations == int(g["iterations"])
    np.testing.assert_allclose(m.density(), g["adjusted"], rtol=1e-13, atol=0)
    assert np.abs(m.fwd_mesh() - g["fwd"]).max() <= POS_TOL
    if m.stats.iterations:
        np.testing.assert_allclose(m.stats.residual, float(g["residual"]), rtol=1e-4, atol=1e-14)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_solve_config1_256_matches_oracle(seed, ot, oracle_port):
    from otmap_b200 import workloads as W

    n = 256
    d = W.to_cells(W.gaussian_mixture(n, seed))
    o = oracle_port.solve(d, n)
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(n)
    m = s.solve(d)
    assert m.stats.iterations == o.iterations
    err = np.abs(m.fwd_mesh() - o.fwd).max()
    assert err <= POS_TOL, err
    assert m.stats.residual <= 1e-7


def test_batch_matches_individual_solves(ot):
    from otmap_b200 import workloads as W

    dens = [W.gaussian_mixture(n, 40 + k) for k, n in enumerate([32, 64, 17, 128, 64])]
    maps = ot.solve_batch(dens)
    for img, m in zip(dens, maps):
        n = img.shape[0]
        s = ot.GridBasedTransportSolver()
        s.set_verbose_level(0)
        s.init(n)
        single = s.solve(W.to_cells(img))
        assert m.stats.iterations == single.stats.iterations
        assert np.array_equal(m.fwd_mesh(), single.fwd_mesh())


@pytest.mark.parametrize("name", golden_names("inverse_"))
def test_inverse_bit_exact(name, ot):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    tm = ot.TransportMap(n, s["fwd"], s["adjusted"])
    pts = np.ascontiguousarray(g["points"].copy())
    face = np.zeros(pts.shape[0], dtype=np.int32)
    nh = np.zeros(pts.shape[0], dtype=np.int32)
    missing = tm.apply_inverse(pts, face, nh)
    assert np.array_equal(nh, g["nhits"])
    assert missing == int((g["nhits"] == 0).sum())
    hit = g["nhits"] > 0
    chosen = chosen_faces(g["faces"], g["nhits"], s["adjusted"])
    assert np.array_equal(face[hit], chosen[hit])
    assert np.array_equal(pts[hit], g["inverse"][hit])


def test_inverse_random_points_1024_shapes(ot, oracle_port):
    """Forward mesh of an oracle solve at 128^2; 2^16 random FP32 points; hit counts,
    located faces and positions bit-exact against the oracle's restatement of the
    reference BVH query, points inside several faces included."""
    from otmap_b200 import workloads as W

    n = 128
    d = W.to_cells(W.blurred_shapes(n, 3, sigma_px=1.0))
    o = oracle_port.solve(d, n, trace=False)
    pts = W.random_points(1 << 16, 7)
    pos_o, face_o, nh_o, _ = oracle_port.apply_inverse(o.fwd, o.density, n, pts)
    tm = ot.TransportMap(n, o.fwd, o.density)
    p = np.ascontiguousarray(pts.copy())
    face = np.zeros(p.shape[0], dtype=np.int32)
    nh = np.zeros(p.shape[0], dtype=np.int32)
    tm.apply_inverse(p, face, nh)
    assert np.array_equal(nh, nh_o)
    assert np.array_equal(face, face_o)
    assert np.array_equal(p, pos_o)


def test_inverse_ties_at_mesh_vertices_and_edges(ot, oracle_port):
    """Points inside several faces: the forward mesh's own vertices (shared by up to four
    faces) and the midpoints of its edges. Hit counts, chosen faces (first hit's weights,
    densest later face, in the reference's BVH order) and positions bit-exact against the
    oracle, and against the reference itself when it is built."""
    from oracle import ref
    from otmap_b200 import workloads as W

    n = 64
    d = W.to_cells(W.gaussian_mixture(n, 12))
    o = oracle_port.solve(d, n)
    V = o.fwd.reshape(n + 1, n + 1, 2)
    mids = np.concatenate([(0.5 * (V[1:, :] + V[:-1, :])).reshape(-1, 2), (0.5 * (V[:, 1:] + V[:, :-1])).reshape(-1, 2)])
    pts = np.ascontiguousarray(np.concatenate([o.fwd, mids]))
    pos_o, face_o, nh_o, _ = oracle_port.apply_inverse(o.fwd, o.density, n, pts)
    assert (nh_o > 1).sum() > 1000  # the case under test
    tm = ot.TransportMap(n, o.fwd, o.density)
    p = pts.copy()
    face = np.zeros(p.shape[0], dtype=np.int32)
    nh = np.zeros(p.shape[0], dtype=np.int32)
    tm.apply_inverse(p, face, nh)
    assert np.array_equal(nh, nh_o)
    assert np.array_equal(face, face_o)
    assert np.array_equal(p, pos_o)
    if ref.available():
        rs = ref.RefSolver()
        rs.init(n)
        rm = rs.solve(d)
        tm2 = ot.TransportMap(n, rm.fwd(), rm.density())
        V2 = rm.fwd().reshape(n + 1, n + 1, 2)
        pts2 = np.ascontiguousarray(np.concatenate([rm.fwd(), (0.5 * (V2[1:, :] + V2[:-1, :])).reshape(-1, 2)]))
        pos_r, _ = rm.apply_inverse(pts2)
        nh_r, _, _ = ref.query_all(rm.fwd(), n, pts2)
        q = pts2.copy()
        nh2 = np.zeros(q.shape[0], dtype=np.int32)
        tm2.apply_inverse(q, None, nh2)
        assert np.array_equal(nh2, nh_r)
        assert np.array_equal(q, pos_r)


@pytest.mark.parametrize("name", golden_names("raster_"))
def test_raster_bit_exact(name, ot):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    for key in g:
        if not key.startswith("img_"):
            continue
        tag, size = key[4:].split("_")
        rows, cols = map(int, size.split("x"))
        img = np.empty((rows, cols))
        ot.rasterize_image(s["fwd"], s["adjusted"] if tag == "dens" else None, img, n=n)
        assert np.array_equal(img, g[key]), key


def test_bad_arguments_raise(ot):
    from otmap_b200 import native

    s = ot.GridBasedTransportSolver()
    with pytest.raises(native.OtmError):
        s._ctx.init(0)
    with pytest.raises(RuntimeError):
        ot.GridBasedTransportSolver().solve(np.ones(16))


@pytest.mark.parametrize("n", [8, 16, 64, 128, 256, 512, 1024, 2048])
def test_fast_and_dense_transforms_agree(n, ot):
    """The fast cosine transform (power-of-two n) and the dense products give the same
    solve: same iterations, positions within 1e-9."""
    from otmap_b200 import native
    from otmap_b200 import workloads as W

    d = W.to_cells(W.gaussian_mixture(n, 70 + n))
    out = {}
    for mode in (native.POISSON_DENSE, native.POISSON_FFT):
        ctx = native.Context(0)
        ctx.set_poisson(mode)
        s = ot.GridBasedTransportSolver(ctx)
        s.set_verbose_level(0)
        s.init(n)
        out[mode] = s.solve(d)
    a, b = out[native.POISSON_DENSE], out[native.POISSON_FFT]
    assert a.stats.iterations == b.stats.iterations
    assert np.abs(a.fwd_mesh() - b.fwd_mesh()).max() <= 1e-9


@pytest.mark.parametrize("n", [2048, 4096])
def test_large_grids_converge(n, ot):
    """Grids above the register transforms' 1024 (the shared-memory FFT of poisson.cu, the
    largest fast-transform sizes): the solve reaches the threshold, the residual recomputed
    from the final mesh (quad areas against e^2 times the adjusted density) is within 2x of
    it, and the map keeps the unit square."""
    from conftest import mesh_residual
    from otmap_b200 import native
    from otmap_b200 import workloads as W

    d = W.to_cells(W.gaussian_mixture(n, 11))
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(n)
    m = s.solve(d)
    assert m.stats.outcome == native.CONVERGED
    assert m.stats.residual <= 1e-7
    fwd = m.fwd_mesh()
    assert mesh_residual(fwd, m.density(), n) <= 2e-7
    assert fwd.min() >= -1e-9 and fwd.max() <= 1 + 1e-9


def test_mixed_batch_uses_both_transforms(ot):
    """A batch mixing power-of-two and other sizes (fast and dense transforms in the
    same launches) matches per-instance solves."""
    from otmap_b200 import workloads as W

    dens = [W.gaussian_mixture(n, 90 + k) for k, n in enumerate([64, 48, 128, 33, 256])]
    maps = ot.solve_batch(dens)
    for img, m in zip(dens, maps):
        n = img.shape[0]
        s = ot.GridBasedTransportSolver()
        s.set_verbose_level(0)
        s.init(n)
        single = s.solve(W.to_cells(img))
        assert m.stats.iterations == single.stats.iterations
        assert np.array_equal(m.fwd_mesh(), single.fwd_mesh())


def test_graph_loop_matches_host_loop(ot):
    """The device-side loop (one CUDA graph launch, WHILE node) and the host-driven loop
    run the same kernels: identical iterations and forward meshes; the graph is reused
    for a second batch of the same sizes and rebuilt for new sizes."""
    from otmap_b200 import native
    from otmap_b200 import workloads as W

    batches = [[W.gaussian_mixture(n, 300 + k) for k, n in enumerate([64, 128, 40, 256])],
               [W.gaussian_mixture(n, 400 + k) for k, n in enumerate([64, 128, 40, 256])],
               [W.gaussian_mixture(n, 500 + k) for k, n in enumerate([32, 512])]]
    results = {}
    for mode in (native.LOOP_GRAPH, native.LOOP_HOST):
        ctx = native.Context(0)
        ctx.set_loop(mode)
        results[mode] = [ot.solve_batch(b, context=ctx) for b in batches]
    for bg, bh in zip(results[native.LOOP_GRAPH], results[native.LOOP_HOST]):
        for mg, mh in zip(bg, bh):
            assert mg.stats.iterations == mh.stats.iterations
            assert mg.stats.outcome == mh.stats.outcome
            assert np.array_equal(mg.fwd_mesh(), mh.fwd_mesh())


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7])
def test_tiny_grids_match_oracle(n, ot, oracle_port):
    """Degenerate sizes: a single cell (already converged), and grids smaller than one
    sweep strip or one transform tile -- same iterations as the oracle, positions within
    1e-6."""
    from otmap_b200 import workloads as W

    d = W.to_cells(W.gaussian_mixture(n, 3)) if n >= 2 else np.ones(1)
    o = oracle_port.solve(d, n)
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(n)
    m = s.solve(d)
    assert m.stats.iterations == o.iterations
    assert np.abs(m.fwd_mesh() - o.fwd).max() <= POS_TOL


def test_batch_outputs_host_and_device_mixed(ot):
    """A batch whose output buffers mix host and device memory: instances that stop early
    have their mesh and density written while the rest still iterate; every output equals
    the one of a single solve."""
    import ctypes as C

    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    sizes = [64, 128, 48, 96]
    dens = [W.to_cells(W.gaussian_mixture(n, 700 + k)) for k, n in enumerate(sizes)]
    ctx = N.Context(0)
    fwd_host = [np.empty(((n + 1) ** 2, 2)) for n in sizes]
    fwd_dev = [torch.empty(((n + 1) ** 2, 2), dtype=torch.float64, device="cuda") for n in sizes]
    adj_host = [np.empty(n * n) for n in sizes]
    fwd_ptrs = [fwd_dev[k].data_ptr() if k % 2 else N.ptr(fwd_host[k]) for k in range(len(sizes))]
    B = len(sizes)
    ns = (C.c_int * B)(*sizes)
    dp = (C.c_void_p * B)(*[N.ptr(d) for d in dens])
    fp = (C.c_void_p * B)(*fwd_ptrs)
    ap = (C.c_void_p * B)(*[N.ptr(a) for a in adj_host])
    stats = (N.SolveStatsC * B)()
    N.check(N.lib().otm_solve_batch(ctx.handle, B, ns, dp, None, fp, ap, stats))
    torch.cuda.synchronize()
    for k, n in enumerate(sizes):
        s = ot.GridBasedTransportSolver()
        s.set_verbose_level(0)
        s.init(n)
        m = s.solve(dens[k])
        got = fwd_dev[k].cpu().numpy() if k % 2 else fwd_host[k]
        assert stats[k].iterations == m.stats.iterations
        assert np.array_equal(got, m.fwd_mesh())
        assert np.array_equal(adj_host[k], m.density())
    ctx.close()


def test_inverse_and_raster_2048(ot, oracle_port):
    """Above the benchmarked size: a GPU-solved 2048^2 map (4.2 M faces), 2^18 FP32-drawn
    query points and the 2048^2 raster. Hit counts and first hits against the reference's
    own BVH (oracle/_ref), positions against the C oracle's apply_inverse_map (pinned to the
    reference's goldens), the raster against the reference's rasterize_image: all
    bit-exact (transport_map.cpp:50-128, rasterizer.cpp:188-236)."""
    from oracle import ref
    from otmap_b200 import workloads as W

    if not ref.available():
        pytest.skip("the reference library (oracle/_ref) is not built")
    n = 2048
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(n)
    m = s.solve(W.to_cells(W.gaussian_mixture(n, 21)))
    fwd, dens = m.fwd_mesh(), m.density()
    pts = W.random_points(1 << 18, 9)
    nh_ref, faces_ref, _ = ref.query_all(fwd, n, pts)
    pos_port, face_port, nh_port, missing_port = oracle_port.apply_inverse(fwd, dens, n, pts)
    assert np.array_equal(nh_port, nh_ref)
    tm = ot.TransportMap(n, fwd, dens)
    p = np.ascontiguousarray(pts.copy())
    face = np.zeros(p.shape[0], dtype=np.int32)
    nh = np.zeros(p.shape[0], dtype=np.int32)
    missing = tm.apply_inverse(p, face, nh)
    assert missing == missing_port == int((nh_ref == 0).sum())
    assert np.array_equal(nh, nh_ref)
    one = nh_ref == 1
    assert np.array_equal(face[one], faces_ref[one, 0])
    assert np.array_equal(face, face_port)
    assert np.array_equal(p, pos_port), int((p != pos_port).any(axis=1).sum())
    img_ref, _ = ref.rasterize(fwd, n, dens, n, n)
    img = np.empty((n, n))
    ot.rasterize_image(fwd, dens, img, n=n)
    assert np.array_equal(img, img_ref), int((img != img_ref).sum())
