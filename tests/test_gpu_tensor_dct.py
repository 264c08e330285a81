"""The tensor-core cosine transform (OTM_POISSON_TENSOR, csrc/dct_tc.cu): the Poisson
solve of otsolver_2dgrid.cpp:175-179 as four tcgen05 products (3xTF32, FP32 accumulation)
for split-precision instances, against the FFT transform of the same mode and against the
FP64 reference's accuracy.

* one iteration from the same start (max_iter = 1): the step taken with the tensor-core
  direction is as close to the step of the FP64 transform as the FFT transform of the same
  mode is (both FP32 transforms; the step's positions and residual differ from the FP64
  step by up to 1e-4 and 7e-4 relative at 1024^2, and the two FP32 forms by about as much);
* whole solves: the reported and the mesh-recomputed residual meet the threshold and the
  map lies within 1e-4 of the FFT-path map;
* a batch mixing tensor-core sizes, FFT sizes and an FP64-only size agrees with single
  solves.
"""

import numpy as np
import pytest

from conftest import mesh_residual

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ot():
    from otmap_b200 import otmap

    return otmap


def solver(ot, poisson):
    from otmap_b200 import native as N

    ctx = N.Context(0)
    ctx.set_precision(N.PRECISION_SPLIT)
    ctx.set_poisson(poisson)
    s = ot.GridBasedTransportSolver(ctx)
    s.set_verbose_level(0)
    return s


@pytest.mark.parametrize("n", [128, 256, 512, 1024])
def test_first_step_matches_fft_transform(n, ot):
    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    d = W.to_cells(W.blurred_shapes(n, 3, sigma_px=n / 200.0))
    opt = ot.SolverOptions(threshold=0.0, max_iter=1)
    f64 = ot.GridBasedTransportSolver(N.Context(0))
    f64.set_verbose_level(0)
    f64.init(n)
    exact = f64.solve(d, opt)
    out = {}
    for mode in (N.POISSON_FFT, N.POISSON_TENSOR):
        s = solver(ot, mode)
        s.init(n)
        out[mode] = s.solve(d, opt)
    a, b = out[N.POISSON_FFT], out[N.POISSON_TENSOR]
    assert exact.stats.iterations == a.stats.iterations == b.stats.iterations == 1
    pos = lambda m: float(np.abs(m.fwd_mesh() - exact.fwd_mesh()).max())
    res = lambda m: abs(m.stats.residual - exact.stats.residual) / exact.stats.residual
    # measured against the FP64 step, FFT / tensor: positions 2.8e-6 / 5.8e-6 (128),
    # 2.5e-5 / 2.7e-5 (256), 6.3e-5 / 6.1e-5 (512), 9.8e-5 / 1.06e-4 (1024); residual
    # 5.6e-6 / 1.7e-5, 1.6e-6 / 3.2e-5, 1.4e-4 / 1.6e-4, 5.2e-4 / 7.2e-4
    assert pos(b) <= 2.0 * pos(a) + 1e-5, (pos(b), pos(a))
    assert res(b) <= 2.0 * res(a) + 1e-4, (res(b), res(a))
    assert float(np.abs(a.fwd_mesh() - b.fwd_mesh()).max()) <= 1e-4


@pytest.mark.parametrize("n", [128, 512])
def test_solve_matches_fft_transform(n, ot):
    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    d = W.to_cells(W.gaussian_mixture(n, 31))
    out = {}
    for mode in (N.POISSON_FFT, N.POISSON_TENSOR):
        s = solver(ot, mode)
        s.init(n)
        out[mode] = s.solve(d)
    a, b = out[N.POISSON_FFT], out[N.POISSON_TENSOR]
    assert b.stats.residual <= 1e-7
    assert mesh_residual(b.fwd_mesh(), b.density(), n) <= 2e-7
    assert abs(a.stats.iterations - b.stats.iterations) <= 3
    assert float(np.abs(a.fwd_mesh() - b.fwd_mesh()).max()) <= 1e-4


def test_batch_mixes_transform_kinds(ot):
    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    sizes = [128, 64, 256, 48, 512]  # tensor, register FFT (64), tensor, FP64 dense (48), tensor
    imgs = [W.gaussian_mixture(n, 950 + k) for k, n in enumerate(sizes)]
    ctx = N.Context(0)
    ctx.set_precision(N.PRECISION_SPLIT)
    ctx.set_poisson(N.POISSON_TENSOR)
    maps = ot.solve_batch(imgs, context=ctx)
    for img, m in zip(imgs, maps):
        n = img.shape[0]
        s = solver(ot, N.POISSON_TENSOR)
        s.init(n)
        single = s.solve(W.to_cells(img))
        assert abs(m.stats.iterations - single.stats.iterations) <= 1
        assert np.abs(m.fwd_mesh() - single.fwd_mesh()).max() <= 1e-6
        assert m.stats.residual <= 1e-7
