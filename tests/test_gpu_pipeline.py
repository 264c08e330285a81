"""Parity of the CUDA rows around the solver (through the C ABI) with the reference's
golden vectors: the PerVertex raster option, triangle and pruned meshes, barycenter
blending and images, transport costs and composite maps. Bit-exact except where the
reference sums sequentially and the GPU in a fixed tree order (costs, image means):
there the tolerance is a few ulps, stated per test."""

import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-13  # sequential vs tree-ordered sums of ~1e3..1e6 positive terms


@pytest.fixture(scope="module")
def ot():
    from otmap_b200 import otmap

    return otmap


@pytest.mark.parametrize("name", golden_names("rasterpv_"))
def test_per_vertex_raster_bit_exact(name, ot):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    for key in g:
        if not key.startswith("img_"):
            continue
        tag, size = key[4:].split("_")
        rows, cols = map(int, size.split("x"))
        dens = s["adjusted"] if tag == "dens" else None
        img = np.empty((rows, cols))
        ot.rasterize_image(s["fwd"], dens, img, ot.RIO_PerVertexDensity, n=n)
        assert np.array_equal(img, g[key]), key
        # the same mesh as an indexed face set takes the general path
        img2 = np.empty((rows, cols))
        ot.rasterize_image(ot.Mesh.grid(n, s["fwd"]), dens, img2, ot.RIO_PerVertexDensity)
        assert np.array_equal(img2, g[key]), key


@pytest.mark.parametrize("name", golden_names("raster_"))
def test_per_face_raster_through_indexed_mesh(name, ot):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    mesh = ot.Mesh.grid(n, s["fwd"])
    for key in g:
        if not key.startswith("img_"):
            continue
        tag, size = key[4:].split("_")
        rows, cols = map(int, size.split("x"))
        img = np.empty((rows, cols))
        ot.rasterize_image(mesh, s["adjusted"] if tag == "dens" else None, img)
        assert np.array_equal(img, g[key]), key


@pytest.mark.parametrize("name", golden_names("meshraster_"))
def test_triangle_and_pruned_mesh_raster_bit_exact(name, ot):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    rows, cols = g["tri_dens_face"].shape
    tri = ot.Mesh(s["fwd"], g["tri_start"], g["tri_idx"])
    pruned = ot.Mesh(g["pruned_xy"], g["pruned_start"], g["pruned_idx"])
    tpruned = ot.Mesh(g["tpruned_xy"], g["tpruned_start"], g["tpruned_idx"])
    for mode, opt in [("face", ot.RIO_PerFaceDensity), ("vertex", ot.RIO_PerVertexDensity)]:
        for mesh, dens, key in [(tri, np.repeat(s["adjusted"], 2), f"tri_dens_{mode}"),
                                (tri, None, f"tri_unit_{mode}"), (pruned, None, f"pruned_unit_{mode}"),
                                (tpruned, None, f"tpruned_unit_{mode}")]:
            img = np.empty((rows, cols))
            ot.rasterize_image(mesh, dens, img, opt)
            assert np.array_equal(img, g[key]), key


def test_mesh_raster_rejects_bad_topology(ot):
    from otmap_b200 import native

    img = np.empty((8, 8))
    bad = ot.Mesh(np.zeros((3, 2)), np.array([0, 3], np.int32), np.array([0, 1, 3], np.int32))
    with pytest.raises(native.OtmError):
        ot.rasterize_image(bad, None, img)
    pent = ot.Mesh(np.zeros((5, 2)), np.array([0, 5], np.int32), np.arange(5, dtype=np.int32))
    with pytest.raises(native.OtmError):
        ot.rasterize_image(pent, None, img)
    empty = ot.Mesh(np.zeros((0, 2)), np.zeros(1, np.int32), np.zeros(0, np.int32))
    ot.rasterize_image(empty, None, img)
    assert not img.any()


def test_barycenter_blend_and_images(ot):
    g = load_golden("barycenter_shapes_n32.npz")
    n = int(g["n"])
    inv = list(g["inv"])
    for k, (a, b) in enumerate(g["pairs"]):
        assert np.array_equal(ot.interpolate(inv, a, b), g[f"mesh_{k}"])
        img, mesh = ot.barycenter_image(inv, a, b, g["means"], n)
        assert np.array_equal(mesh, g[f"mesh_{k}"])
        np.testing.assert_allclose(img, g[f"img_{k}"], rtol=SUM_RTOL, atol=0)
    for k, a in enumerate(g["lalphas"]):
        assert np.array_equal(ot.interpolate(inv[:2], a), g[f"lmesh_{k}"])
        img, _ = ot.barycenter_image(inv[:2], a, None, g["means"][:2], n)
        np.testing.assert_allclose(img, g[f"limg_{k}"], rtol=SUM_RTOL, atol=0)


def test_barycenter_pipeline_from_densities(ot):
    """The whole demo on the GPU: batched solves of the four densities, inverse of the
    grid vertices, one barycenter image whose mean is the blended density mean."""
    g = load_golden("barycenter_shapes_n32.npz")
    n = int(g["n"])
    maps = ot.solve_batch(list(g["images"]))
    inv = []
    for k, m in enumerate(maps):
        assert np.abs(m.fwd_mesh() - g["fwd"][k]).max() <= 1e-6
        pts = ot.grid_vertices(n)
        nh = np.zeros(pts.shape[0], dtype=np.int32)
        m.apply_inverse(pts, None, nh)
        assert (nh >= 1).all()
        assert np.abs(pts - g["inv"][k]).max() <= 1e-4
        inv.append(pts)
    img, _ = ot.barycenter_image(inv, 0.25, 0.5, g["means"], n)
    assert np.isfinite(img).all()
    np.testing.assert_allclose(img.mean(), float(g["expected_1"]), rtol=1e-12)


def test_inverse_fast_mode_agrees_on_single_hits(ot):
    s = load_golden("solve_mix_n64_s1.npz")
    g = load_golden("inverse_mix_n64_s1.npz")
    tm = ot.TransportMap(64, s["fwd"], s["adjusted"])
    a = np.ascontiguousarray(g["points"].copy())
    b = a.copy()
    nh = np.zeros(a.shape[0], dtype=np.int32)
    tm.apply_inverse(a, None, nh)
    tm.apply_inverse(b, fast=True)
    one = nh == 1
    assert np.array_equal(a[one], b[one])
    assert np.array_equal(b[one], g["inverse"][one])


@pytest.mark.parametrize("name", golden_names("cost_"))
def test_transport_cost_matches_reference(name, ot):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    c, pf = ot.transport_cost(ot.grid_vertices(n), s["fwd"], s["adjusted"], cost_per_face=True)
    np.testing.assert_allclose(c, float(g["cost"]), rtol=SUM_RTOL, atol=0)
    np.testing.assert_allclose(pf, g["per_face"], rtol=SUM_RTOL, atol=0)
    assert ot.transport_cost(ot.grid_vertices(n), s["fwd"], s["adjusted"]) == c


def test_composite_maps_and_costs(ot):
    g = load_golden("compose_mix_n32_n37.npz")
    u = load_golden(str(g["u"]) + ".npz")
    v = load_golden(str(g["v"]) + ".npz")
    tu = ot.TransportMap(int(u["n"]), u["fwd"], u["adjusted"])
    tv = ot.TransportMap(int(v["n"]), v["fwd"], v["adjusted"])
    uv, vu = ot.compose(tu, tv), ot.compose(tv, tu)
    one = g["nhits_uv"] == 1
    assert np.array_equal(uv[one], g["map_uv"][one])
    one = g["nhits_vu"] == 1
    assert np.array_equal(vu[one], g["map_vu"][one])
    c = ot.transport_cost(ot.grid_vertices(int(u["n"])), uv, u["adjusted"])
    np.testing.assert_allclose(c, float(g["cost_uv"]), rtol=SUM_RTOL)
    c = ot.transport_cost(ot.grid_vertices(int(v["n"])), vu, v["adjusted"])
    np.testing.assert_allclose(c, float(g["cost_vu"]), rtol=SUM_RTOL)


def test_large_transport_cost_against_oracle(ot, oracle_port):
    """1024^2 grid, a smooth displacement and a random density: GPU cost vs the
    oracle's sequential restatement."""
    n = 1024
    rng = np.random.default_rng(11)
    src = ot.grid_vertices(n)
    dst = src + 0.01 * np.sin(7 * src[:, ::-1] + rng.random(2))
    dens = rng.random(n * n) + 0.1
    c_o = oracle_port.transport_cost(src, dst, dens, n)
    c, pf = ot.transport_cost(src, dst, dens, cost_per_face=True)
    np.testing.assert_allclose(c, c_o, rtol=1e-12)
    assert np.isfinite(pf).all()
    np.testing.assert_allclose(pf.sum(), c, rtol=1e-12)


@pytest.mark.parametrize("kind", ["grid", "tri", "pruned"])
def test_splat_matches_oracle_bit_exact(ot, oracle_port, kind):
    """The GPU splat and the oracle use the same counter-based generator: identical
    counts on grid, triangle and pruned meshes, for two seeds."""
    g = load_golden("meshraster_mix_n32_s0.npz")
    s = load_golden("solve_mix_n32_s0.npz")
    n = 32
    st, ix = oracle_port.grid_faces(n)
    if kind == "grid":
        mesh, xy = s["fwd"], s["fwd"]
    elif kind == "tri":
        st, ix = g["tri_start"], g["tri_idx"]
        mesh, xy = ot.Mesh(s["fwd"], st, ix), s["fwd"]
    else:
        st, ix, xy = g["pruned_start"], g["pruned_idx"], g["pruned_xy"]
        mesh = ot.Mesh(xy, st, ix)
    nf = st.size - 1
    rng = np.random.default_rng(4)
    spf = rng.integers(0, 400, nf).astype(np.int32)
    for seed in (0, 12345678901):
        img = np.empty((n + 3, n))
        ot.sample_transportmap_to_image(mesh, spf, img, seed)
        want = oracle_port.sample_image(xy, st, ix, spf, seed, n + 3, n)
        assert np.array_equal(img, want), (kind, seed)


def test_splat_large_grid_counts(ot):
    """1024^2 origin grid, 300 samples per face into a 1024^2 image: every pixel gets
    exactly its face's 300 samples (3.1e8 samples)."""
    n = 1024
    img = np.empty((n, n))
    ot.sample_transportmap_to_image(ot.grid_vertices(n), 300, img, 9)
    assert img.sum() == 300.0 * n * n
    assert (img == 300).mean() > 0.9999


def test_synthetize_image_scales(ot):
    s = load_golden("solve_mix_n32_s0.npz")
    sampled, raster = ot.synthetize_image(s["fwd"], 32, s["density"], s["adjusted"], samples_per_face=100, seed=5)
    np.testing.assert_allclose(sampled.sum(), s["density"].sum(), rtol=1e-2)
    assert np.isfinite(raster).all() and raster.max() > 0


@pytest.mark.parametrize("name", golden_names("gridcost_"))
def test_solver_transport_cost_matches_reference(name, ot):
    """compute_transport_cost: per-face values bit-exact, the sum to a few ulps."""
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    total, pf = ot.grid_transport_cost(g["grads"], s["adjusted"], per_face=True)
    assert np.array_equal(pf, g["per_face"])
    np.testing.assert_allclose(total, float(g["total"]), rtol=SUM_RTOL)


def test_device_tensors_through_inversion_and_barycenters(ot):
    """The same pipeline with the points and inverse meshes held as CUDA tensors (device
    pointers through the C ABI): inverse positions and images bitwise equal to the numpy
    path; maps destroyed and rebuilt in a loop reuse the stream-ordered pool."""
    import torch

    from otmap_b200 import workloads as W

    n = 64
    dens = [W.gaussian_mixture(n, 40 + k) for k in range(4)]
    maps = ot.solve_batch(dens)
    inv_h, inv_d = [], []
    for m in maps:
        p = ot.grid_vertices(n).copy()
        m.apply_inverse(p)
        inv_h.append(p)
        q = torch.from_numpy(ot.grid_vertices(n)).cuda()
        m.apply_inverse(q)
        inv_d.append(q)
        assert np.array_equal(q.cpu().numpy(), p)
    means = [W.to_cells(d).mean() for d in dens]
    img_h, mesh_h = ot.barycenter_image(inv_h, 0.3, 0.6, means, 96)
    img_d, mesh_d = ot.barycenter_image(inv_d, 0.3, 0.6, means, 96, want_mesh=False)
    assert mesh_d is None
    assert np.array_equal(img_h, img_d)
    blend = ot.interpolate(inv_d, 0.3, 0.6)
    assert np.array_equal(blend, mesh_h)
    for _ in range(20):  # create, locate, destroy: buffers come back from the pool
        m = ot.TransportMap(n, maps[0].fwd_mesh(), maps[0].density())
        r = ot.grid_vertices(n).copy()
        m.apply_inverse(r)
        m.release()
        assert np.array_equal(r, inv_h[0])
