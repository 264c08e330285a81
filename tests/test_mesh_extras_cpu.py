"""CPU checks of the rows around the solver: the oracle against the reference's golden
vectors for the PerVertex raster option, triangle and pruned meshes, barycenter
blending and composite-map costs; and the library's host-side mesh code (grid faces,
prune_empty_faces, OFF read/write), which needs no GPU, against the same goldens and
against the reference library itself where it is built."""

import os
import struct

import numpy as np
import pytest

from conftest import golden_names, load_golden


def _ref():
    from oracle import ref

    if not ref.available():
        pytest.skip("reference library not built")
    return ref


@pytest.fixture(scope="module")
def ot():
    from otmap_b200 import build, native, otmap

    if not os.path.exists(native.LIB_PATH):
        build.build_library()
    return otmap


# ---- oracle vs reference goldens ----

@pytest.mark.parametrize("name", golden_names("rasterpv_"))
def test_oracle_per_vertex_raster(name, oracle_port):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    st, ix = oracle_port.grid_faces(n)
    for key in g:
        if not key.startswith("img_"):
            continue
        tag, size = key[4:].split("_")
        rows, cols = map(int, size.split("x"))
        img = oracle_port.rasterize_mesh(s["fwd"], st, ix, s["adjusted"] if tag == "dens" else None, rows, cols,
                                         per_vertex=True)
        assert np.array_equal(img, g[key]), key


@pytest.mark.parametrize("name", golden_names("meshraster_"))
def test_oracle_triangle_and_pruned_meshes(name, oracle_port):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    st, ix = oracle_port.grid_faces(n)
    pxy, pst, pix = oracle_port.prune_empty_faces(s["fwd"], st, ix, g["zeroed"])
    assert np.array_equal(pxy, g["pruned_xy"]) and np.array_equal(pst, g["pruned_start"])
    assert np.array_equal(pix, g["pruned_idx"])
    txy, tst, tix = oracle_port.prune_empty_faces(s["fwd"], g["tri_start"], g["tri_idx"], g["zeroed"])
    assert np.array_equal(txy, g["tpruned_xy"]) and np.array_equal(tix, g["tpruned_idx"])
    rows, cols = g["tri_dens_face"].shape
    for mode, pv in [("face", False), ("vertex", True)]:
        img = oracle_port.rasterize_mesh(s["fwd"], g["tri_start"], g["tri_idx"], np.repeat(s["adjusted"], 2), rows,
                                         cols, per_vertex=pv)
        assert np.array_equal(img, g[f"tri_dens_{mode}"])
        img = oracle_port.rasterize_mesh(pxy, pst, pix, None, rows, cols, per_vertex=pv)
        assert np.array_equal(img, g[f"pruned_unit_{mode}"])
        img = oracle_port.rasterize_mesh(txy, tst, tix, None, rows, cols, per_vertex=pv)
        assert np.array_equal(img, g[f"tpruned_unit_{mode}"])


def test_oracle_barycenter_blend(oracle_port):
    g = load_golden("barycenter_shapes_n32.npz")
    inv = list(g["inv"])
    for k, (a, b) in enumerate(g["pairs"]):
        w = [(1. - a) * (1. - b), a * (1. - b), a * b, (1. - a) * b]
        assert np.array_equal(oracle_port.mesh_blend(inv, w), g[f"mesh_{k}"])
    for k, a in enumerate(g["lalphas"]):
        assert np.array_equal(oracle_port.mesh_blend(inv[:2], [1. - a, a]), g[f"lmesh_{k}"])


def test_oracle_composite_costs(oracle_port):
    g = load_golden("compose_mix_n32_n37.npz")
    u = load_golden(str(g["u"]) + ".npz")
    v = load_golden(str(g["v"]) + ".npz")
    c = oracle_port.transport_cost(oracle_port.grid_vertices(int(u["n"])), g["map_uv"], u["adjusted"], int(u["n"]))
    assert c == float(g["cost_uv"])
    c = oracle_port.transport_cost(oracle_port.grid_vertices(int(v["n"])), g["map_vu"], v["adjusted"], int(v["n"]))
    assert c == float(g["cost_vu"])


# ---- the library's host-side mesh code ----

def test_grid_faces_match_oracle(ot, oracle_port):
    for n in (1, 2, 7, 32):
        m = ot.Mesh.grid(n)
        st, ix = oracle_port.grid_faces(n)
        assert np.array_equal(m.face_start, st) and np.array_equal(m.face_vertices, ix)


@pytest.mark.parametrize("name", golden_names("meshraster_"))
def test_library_prune_matches_reference(name, ot):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    p = ot.prune_empty_faces(s["fwd"], g["zeroed"])
    assert np.array_equal(p.xy, g["pruned_xy"])
    assert np.array_equal(p.face_start, g["pruned_start"]) and np.array_equal(p.face_vertices, g["pruned_idx"])
    tri = ot.Mesh(s["fwd"].copy(), g["tri_start"], g["tri_idx"])
    p = ot.prune_empty_faces(tri, g["zeroed"])
    assert np.array_equal(p.xy, g["tpruned_xy"])
    assert np.array_equal(p.face_start, g["tpruned_start"]) and np.array_equal(p.face_vertices, g["tpruned_idx"])


def test_prune_edge_cases(ot, oracle_port):
    n = 6
    xy = ot.grid_vertices(n)
    st, ix = oracle_port.grid_faces(n)
    for dens in (np.ones(n * n), np.zeros(n * n), np.r_[np.zeros(n * n - 1), 1.0], np.r_[1.0, np.zeros(n * n - 1)]):
        p = ot.prune_empty_faces(xy, dens)
        q = oracle_port.prune_empty_faces(xy, st, ix, dens)
        assert np.array_equal(p.xy, q[0]) and np.array_equal(p.face_start, q[1])
        assert np.array_equal(p.face_vertices, q[2])
    assert ot.prune_empty_faces(xy, np.zeros(n * n)).n_faces == 0


def test_prune_matches_reference_random(ot, oracle_port):
    ref = _ref()
    rng = np.random.default_rng(3)
    n = 20
    xy = ot.grid_vertices(n) + rng.normal(0, 1e-3, ((n + 1) ** 2, 2))
    st, ix = oracle_port.grid_faces(n)
    for frac in (0.1, 0.5, 0.9):
        dens = np.where(rng.random(n * n) < frac, 0.0, 1.0)
        a = ref.prune_empty_faces(xy, st, ix, dens)
        b = ot.prune_empty_faces(xy, dens)
        assert np.array_equal(a[0], b.xy) and np.array_equal(a[1], b.face_start)
        assert np.array_equal(a[2], b.face_vertices)


def test_off_written_byte_for_byte(ot, tmp_path):
    ref = _ref()
    g = load_golden("meshraster_mix_n32_s0.npz")
    s = load_golden("solve_mix_n32_s0.npz")
    meshes = [ot.Mesh.grid(32, s["fwd"]), ot.Mesh(g["pruned_xy"], g["pruned_start"], g["pruned_idx"]),
              ot.Mesh(g["tpruned_xy"], g["tpruned_start"], g["tpruned_idx"]),
              ot.Mesh(np.array([[-0.0, 1e-12], [123.456, -7.0]]), np.zeros(1, np.int32), np.zeros(0, np.int32))]
    for k, m in enumerate(meshes):
        a, b = tmp_path / f"ref{k}.off", tmp_path / f"ours{k}.off"
        ref.write_off(a, m.xy, m.face_start, m.face_vertices)
        m.write(str(b))
        assert a.read_bytes() == b.read_bytes(), k
    ot.write_off(str(tmp_path / "grid.off"), s["fwd"])
    assert (tmp_path / "grid.off").read_bytes() == (tmp_path / "ref0.off").read_bytes()


def test_off_read_matches_reference(ot, tmp_path):
    ref = _ref()
    g = load_golden("meshraster_shapes_n64_s5.npz")
    m = ot.Mesh(g["tpruned_xy"], g["tpruned_start"], g["tpruned_idx"])
    path = tmp_path / "m.off"
    m.write(str(path))
    r = ot.Mesh.read(str(path))
    a = ref.read_off(path, m.n_vertices, m.n_faces, m.face_vertices.size)
    assert np.array_equal(r.xy, a[0]) and np.array_equal(r.face_start, a[1]) and np.array_equal(r.face_vertices, a[2])
    assert np.abs(r.xy - m.xy).max() <= 5e-11  # "%.10f" rounding
    assert np.array_equal(r.face_vertices, m.face_vertices)
    # headers with per-vertex normals / colours, and the binary form
    (tmp_path / "n.off").write_text("NOFF\n3 1 0\n0.5 0.25 0 0 0 1\n1 0 0 0 0 1\n0 1 0 0 0 1\n3 0 1 2\n")
    (tmp_path / "c.off").write_text("COFF\n3 1 0\n0.5 0.25 0 255 0 0\n1 0 0 0 255 0\n0 1 0 0 0 255\n3 2 1 0\n")
    blob = b"OFF BINARY\n" + struct.pack("<3I", 4, 1, 0)
    for p in [(0.1, 0.2, 0.0), (0.9, 0.2, 0.0), (0.9, 0.8, 0.0), (0.1, 0.8, 0.0)]:
        blob += struct.pack("<3d", *p)
    blob += struct.pack("<5I", 4, 0, 1, 2, 3)
    (tmp_path / "b.off").write_bytes(blob)
    for f in ("n.off", "c.off", "b.off"):
        r = ot.Mesh.read(str(tmp_path / f))
        a = ref.read_off(tmp_path / f, 8, 8, 8)
        assert np.array_equal(r.xy, a[0]) and np.array_equal(r.face_start, a[1]), f
        assert np.array_equal(r.face_vertices, a[2]), f


def test_mesh_io_rejects_bad_input(ot, tmp_path):
    from otmap_b200 import native

    with pytest.raises(native.OtmError):
        ot.Mesh.read(str(tmp_path / "missing.off"))
    (tmp_path / "bad.off").write_text("PLY\n")
    with pytest.raises(native.OtmError):
        ot.Mesh.read(str(tmp_path / "bad.off"))
    (tmp_path / "oob.off").write_text("OFF\n3 1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 7\n")
    with pytest.raises(native.OtmError):
        ot.Mesh.read(str(tmp_path / "oob.off"))
    bad = ot.Mesh(np.zeros((3, 2)), np.array([0, 3], np.int32), np.array([0, 1, 5], np.int32))
    with pytest.raises(native.OtmError):
        bad.write(str(tmp_path / "x.off"))
    with pytest.raises(native.OtmError):
        ot.prune_empty_faces(bad, np.ones(1))


# ---- stochastic splat: the oracle's generator vs the reference's std::rand() ----

def _zscores(a, b):
    return (a - b) / np.sqrt(a + b + 1.0)


@pytest.mark.parametrize("tri", [False, True])
def test_oracle_splat_matches_reference_in_distribution(oracle_port, tri):
    """Same mesh, same samples per face: the two images differ only by sampling noise
    (per-pixel z-scores of the difference are O(1)) and count the same points."""
    ref = _ref()
    g = load_golden("solve_mix_n32_s0.npz")
    n = 32
    st, ix = oracle_port.grid_faces(n)
    if tri:
        q = ix.reshape(-1, 4)
        ix = np.stack([q[:, [0, 1, 2]], q[:, [0, 2, 3]]], 1).reshape(-1).astype(np.int32)
        st = np.arange(0, ix.size + 1, 3, dtype=np.int32)
    nf = st.size - 1
    spf = np.full(nf, 1500, np.int32)
    spf[::7] = 300
    a = ref.sample_image(g["fwd"], st, ix, spf, 1, n + 5, n)
    b = oracle_port.sample_image(g["fwd"], st, ix, spf, 1, n + 5, n)
    assert a.sum() == b.sum() == spf.sum()
    z = _zscores(a, b)
    assert np.abs(z).max() < 5.0 and z.std() < 1.3


def test_oracle_splat_on_the_origin_grid_is_exact(oracle_port):
    """On the undeformed grid each face is one pixel: every pixel counts its face's samples."""
    n = 16
    st, ix = oracle_port.grid_faces(n)
    t = np.arange(n + 1) / n
    xy = np.stack([np.repeat(t, n + 1), np.tile(t, n + 1)], 1)
    spf = (np.arange(n * n) % 5 + 1).astype(np.int32) * 10
    img = oracle_port.sample_image(xy, st, ix, spf, 3, n, n)
    want = spf.reshape(n, n).T  # face f = j + i*n covers pixel (row j, col i)
    assert np.array_equal(img, want)


@pytest.mark.parametrize("name", golden_names("gridcost_"))
def test_oracle_solver_transport_cost(name, oracle_port):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    c, pf = oracle_port.grid_transport_cost(g["grads"], s["adjusted"], int(g["n"]))
    assert np.array_equal(pf, g["per_face"])
    np.testing.assert_allclose(c, float(g["total"]), rtol=1e-14)
