"""CPU checks of the reference-gradient builder used by the GPU adjoint tests."""

import numpy as np


def test_jacobian_at_rest_is_minus_pseudo_laplacian(oracle_port):
    from adjoint_ref import area_jacobian, grad_operator

    n = 12
    t = np.arange(n + 1) / n
    grid = np.stack([np.repeat(t, n + 1), np.tile(t, n + 1)], axis=1)
    J = (area_jacobian(grid, n) @ grad_operator(n)).toarray()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(n * n)
    np.testing.assert_allclose(J @ x, -oracle_port.laplacian_apply(x, n), atol=1e-12)


def test_jacobian_matches_finite_difference_of_areas(oracle_port):
    from adjoint_ref import area_jacobian, grad_operator
    from otmap_b200 import workloads as W

    n = 10
    d = W.to_cells(W.gaussian_mixture(n, 3))
    o = oracle_port.solve(d, n)
    J = (area_jacobian(o.fwd, n) @ grad_operator(n)).toarray()
    rng = np.random.default_rng(1)
    u = rng.standard_normal(n * n)
    h = 1e-6
    rp, _ = oracle_port.residual(o.psi + h * u, o.density, n)
    rm, _ = oracle_port.residual(o.psi - h * u, o.density, n)
    np.testing.assert_allclose(J @ u, (rp - rm) / (2 * h), rtol=1e-6, atol=1e-12)
