"""The C++ facade (namespace otmap over the C ABI) on the GPU: the calls of the
reference's demo apps/otmap.cpp (solve two maps, costs, inverse meshes, composite maps,
raster, prune, OFF output) made from C++, checked against the reference's golden
vectors and against the same calls through the Python API."""

import subprocess

import numpy as np
import pytest

import facade_build
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _write_density(path, n, d):
    with open(path, "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(np.ascontiguousarray(d, dtype=np.float64).tobytes())


def _f64(path, shape=None):
    a = np.fromfile(path, dtype=np.float64)
    return a.reshape(shape) if shape else a


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    return facade_build.build(str(tmp_path_factory.mktemp("facade")))


def _run(exe, folder, gu, gv):
    _write_density(folder / "u.bin", int(gu["n"]), gu["density"])
    _write_density(folder / "v.bin", int(gv["n"]), gv["density"])
    r = subprocess.run([exe, "pipeline", str(folder), str(folder / "u.bin"), str(folder / "v.bin")],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    assert r.returncode == 0, r.stdout
    return facade_build.results(str(folder))


def test_facade_pipeline_matches_reference_and_python(exe, tmp_path):
    from otmap_b200 import otmap as ot

    gu, gv = load_golden("solve_mix_n32_s0.npz"), load_golden("solve_mix_n37_s10.npz")
    comp = load_golden("compose_mix_n32_n37.npz")
    res = _run(exe, tmp_path, gu, gv)
    nu, nv = int(gu["n"]), int(gv["n"])
    assert res["iterations_u"] == int(gu["iterations"]) and res["iterations_v"] == int(gv["iterations"])
    fu = _f64(tmp_path / "u_fwd.f64", (-1, 2))
    fv = _f64(tmp_path / "v_fwd.f64", (-1, 2))
    assert np.abs(fu - gu["fwd"]).max() <= 1e-6 and np.abs(fv - gv["fwd"]).max() <= 1e-6
    # the same library through Python gives the same bits
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(nu)
    mu = s.solve(gu["density"])
    s.init(nv)
    mv = s.solve(gv["density"])
    assert np.array_equal(fu, mu.fwd_mesh()) and np.array_equal(fv, mv.fwd_mesh())
    assert np.array_equal(_f64(tmp_path / "u_density.f64"), mu.density())
    assert res["cost_u"] == ot.transport_cost(ot.grid_vertices(nu), mu.fwd_mesh(), mu.density())
    inv = ot.grid_vertices(nu)
    ot.apply_inverse_map(mu, inv, 0)
    assert np.array_equal(_f64(tmp_path / "u_inv.f64", (-1, 2)), inv)
    ot.write_off(str(tmp_path / "py_u_fwd.off"), mu.fwd_mesh())
    assert (tmp_path / "py_u_fwd.off").read_bytes() == (tmp_path / "u_fwd.off").read_bytes()
    # composite map u -> v against the reference, from the reference's own meshes
    tu = ot.TransportMap(nu, gu["fwd"], gu["adjusted"])
    tv = ot.TransportMap(nv, gv["fwd"], gv["adjusted"])
    uv_ref_inputs = ot.compose(tu, tv)
    one = comp["nhits_uv"] == 1
    assert np.array_equal(uv_ref_inputs[one], comp["map_uv"][one])
    uv = ot.compose(mu, mv)
    assert np.array_equal(_f64(tmp_path / "map_uv.f64", (-1, 2)), uv)
    np.testing.assert_allclose(res["cost_uv"], float(comp["cost_uv"]), rtol=1e-6)
    img = np.empty((nu, nu))
    ot.rasterize_image(uv, None, img)
    assert np.array_equal(_f64(tmp_path / "map_uv_raster.f64", (nu, nu)), img)
    img = np.empty((nu, nu))
    ot.rasterize_image(uv, mu.density(), img, ot.RIO_PerVertexDensity)
    assert np.array_equal(_f64(tmp_path / "map_uv_pervertex.f64", (nu, nu)), img)
    pr = ot.prune_empty_faces(uv, mu.density())
    pr.write(str(tmp_path / "py_map_uv.off"))
    assert (tmp_path / "py_map_uv.off").read_bytes() == (tmp_path / "map_uv.off").read_bytes()
    img = np.empty((nu + 3, nu))
    ot.rasterize_image(pr, None, img)
    assert np.array_equal(_f64(tmp_path / "map_uv_pruned_raster.f64", (nu + 3, nu)), img)
    q = mv.inv([0.37, 0.61])
    assert (res["inv_x"], res["inv_y"]) == (q[0], q[1])
    img = np.empty((nu, nu))
    ot.sample_transportmap_to_image(mu.fwd_mesh(), 50, img, 7)
    assert np.array_equal(_f64(tmp_path / "u_fwd_samples.f64", (nu, nu)), img)
    for tag, m in (("u", mu), ("v", mv)):
        assert np.array_equal(_f64(tmp_path / f"batch_{tag}_fwd.f64", (-1, 2)), m.fwd_mesh())


def test_facade_linear_barycenter(exe, tmp_path):
    from otmap_b200 import otmap as ot

    gu, gv = load_golden("solve_mix_n32_s0.npz"), load_golden("solve_mix_n32_s7_iter5.npz")
    _run(exe, tmp_path, gu, gv)
    maps = []
    s = ot.GridBasedTransportSolver()
    s.set_verbose_level(0)
    s.init(32)
    for g in (gu, gv):
        m = s.solve(g["density"])
        p = ot.grid_vertices(32)
        ot.apply_inverse_map(m, p, 0)
        maps.append(p)
    assert np.array_equal(_f64(tmp_path / "mid.f64", (-1, 2)), ot.interpolate(maps, 0.5))
