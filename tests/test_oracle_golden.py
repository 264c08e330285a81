"""Pins the C restatement of the reference (oracle/otmap_oracle.c) against the golden
vectors the reference itself produced (tests/golden/make_golden.py)."""

import numpy as np
import pytest

from conftest import golden_names, load_golden


@pytest.mark.parametrize("name", golden_names("solve_"))
def test_solve_matches_reference(name, oracle_port):
    g = load_golden(name)
    n = int(g["n"])
    o = oracle_port.solve(g["density"], n, beta_cj=bool(g["beta_cj"]), max_iter=int(g["max_iter"]),
                          threshold=float(g["threshold"]), max_ratio=float(g["max_ratio"]))
    assert o.iterations == int(g["iterations"])
    np.testing.assert_allclose(o.density, g["adjusted"], rtol=1e-13, atol=0)
    # vertex positions: the oracle and the reference differ only in the Laplacian solve's rounding
    assert np.abs(o.fwd - g["fwd"]).max() <= 1e-10
    if o.iterations:
        np.testing.assert_allclose(o.trace[:, 0], g["trace"][:, 0], rtol=1e-8, atol=1e-12)  # alpha
        np.testing.assert_allclose(o.trace[:, 1], g["trace"][:, 1], rtol=1e-7, atol=1e-10)  # beta
        np.testing.assert_allclose(o.trace[:, 3], g["trace"][:, 3], rtol=1e-5, atol=1e-14)  # res^2
    np.testing.assert_allclose(o.residual, float(g["residual"]), rtol=1e-5, atol=1e-14)


@pytest.mark.parametrize("name", golden_names("units_"))
def test_protected_steps_match_reference(name, oracle_port):
    g = load_golden(name)
    n = int(g["n"])
    P = oracle_port
    np.testing.assert_allclose(P.vertex_gradients(g["psi"], n), g["grads"], rtol=0, atol=1e-15)
    r, res = P.residual(g["psi"], g["density"], n)
    np.testing.assert_allclose(r, g["r"], rtol=0, atol=1e-16)
    np.testing.assert_allclose(res, float(g["res"]), rtol=1e-12)
    lap = P.poisson_dct(g["rhs"], n)
    np.testing.assert_allclose(lap, g["lap"], rtol=0, atol=1e-10 * np.abs(g["lap"]).max())
    g0 = P.vertex_gradients(g["psi"], n)
    gd = P.vertex_gradients(g["direction"], n)
    a, b = P.line_params(g0, gd, n)
    np.testing.assert_allclose(a, g["a"], rtol=0, atol=1e-16)
    np.testing.assert_allclose(b, g["b"], rtol=0, atol=1e-16)


@pytest.mark.parametrize("name", golden_names("inverse_"))
def test_inverse_bit_exact(name, oracle_port):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    pos, faces, nh, missing = oracle_port.apply_inverse(s["fwd"], s["adjusted"], n, g["points"])
    assert np.array_equal(nh, g["nhits"])
    ok = nh > 0
    assert np.array_equal(pos[ok], g["inverse"][ok])
    nhq, fq, bq = oracle_port.query_all(s["fwd"], n, g["points"], cap=2)
    assert np.array_equal(fq, g["faces"])
    assert np.array_equal(bq[:, 0], g["bary"])


@pytest.mark.parametrize("name", golden_names("raster_"))
def test_raster_bit_exact(name, oracle_port):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    for key in g:
        if not key.startswith("img_"):
            continue
        tag, size = key[4:].split("_")
        rows, cols = map(int, size.split("x"))
        dens = s["adjusted"] if tag == "dens" else None
        img = oracle_port.rasterize(s["fwd"], n, dens, rows, cols, stale_weights=True)
        assert np.array_equal(img, g[key]), key


@pytest.mark.parametrize("name", golden_names("cost_"))
def test_transport_cost_bit_exact(name, oracle_port):
    g = load_golden(name)
    s = load_golden(str(g["solve"]) + ".npz")
    n = int(g["n"])
    c, pf = oracle_port.transport_cost(oracle_port.grid_vertices(n), s["fwd"], s["adjusted"], n, per_face=True)
    assert c == float(g["cost"])
    assert np.array_equal(pf, g["per_face"])
