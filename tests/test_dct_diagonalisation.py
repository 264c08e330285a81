"""The assembled pseudo-Laplacian of otsolver_2dgrid.cpp:284-311 is diagonalised by the
orthonormal 2-D DCT-II, and the pinned solve + mean projection of :175-179 equals the
DCT pseudo-inverse. The GPU Poisson solve relies on both facts."""

import numpy as np
import pytest

import dct_tables as dct


@pytest.mark.parametrize("n", [1, 2, 3, 8, 17, 32, 64])
def test_matrix_is_diagonalised(n, oracle_port):
    rng = np.random.default_rng(n)
    C = dct.basis(n)
    lam = dct.eigenvalues(n)
    for _ in range(3):
        x = rng.standard_normal(n * n)
        y = oracle_port.laplacian_apply(x, n)
        X = x.reshape(n, n)
        y2 = (C.T @ (lam * (C @ X @ C.T)) @ C).ravel()
        assert np.abs(y - y2).max() <= 1e-13 * max(1.0, np.abs(y).max())


@pytest.mark.parametrize("n", [4, 9, 16, 24])
def test_pinned_solve_equals_pseudo_inverse(n, oracle_port):
    rng = np.random.default_rng(100 + n)
    r = rng.standard_normal(n * n)
    r -= r.mean()
    d_pin = oracle_port.poisson_pinned(r, n)
    d_dct = oracle_port.poisson_dct(r, n)
    assert np.abs(d_pin - d_dct).max() <= 1e-10 * np.abs(d_dct).max()


def test_basis_orthonormal():
    for n in (1, 5, 64):
        C = dct.basis(n)
        assert np.abs(C @ C.T - np.eye(n)).max() < 1e-13
