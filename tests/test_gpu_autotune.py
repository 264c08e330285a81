"""OTM_OPT_AUTOTUNE: the sweeps' strip height of a batch configuration is timed on the
first call (16, 32, 64 rows) and kept; the tuned solve starts from the same state as an
untuned one, so it reaches the same map up to the order of the partial sums, and a
second call of the configuration reuses the choice (no new timing: bitwise the same
result)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotuned_batch_matches_untuned():
    from otmap_b200 import native as N
    from otmap_b200 import otmap as ot
    from otmap_b200 import workloads as W

    imgs = [W.gaussian_mixture(n, 700 + k) for k, n in enumerate([128, 256, 512, 1024, 64])]
    for prec in (N.PRECISION_FP64, N.PRECISION_SPLIT):
        plain = N.Context(0)
        plain.set_precision(prec)
        ref = ot.solve_batch(imgs, context=plain)
        rule = plain.strip_rows()
        assert rule in (16, 32, 64)
        tuned = N.Context(0)
        tuned.set_precision(prec)
        tuned.set_autotune(True)
        assert tuned.get_option(N.OPT_AUTOTUNE) == N.AUTOTUNE_ON
        first = ot.solve_batch(imgs, context=tuned)
        rows = tuned.strip_rows()
        assert rows in (16, 32, 64)
        second = ot.solve_batch(imgs, context=tuned)
        assert tuned.strip_rows() == rows
        tol = 1e-8 if prec == N.PRECISION_FP64 else 1e-5
        for a, b, c in zip(ref, first, second):
            assert abs(a.stats.iterations - b.stats.iterations) <= 1
            assert np.abs(a.fwd_mesh() - b.fwd_mesh()).max() <= tol
            assert b.stats.iterations == c.stats.iterations
            assert np.array_equal(b.fwd_mesh(), c.fwd_mesh())
            assert np.array_equal(b.density(), a.density())  # the tuning runs leave the densities as given


def test_autotune_option_validation():
    from otmap_b200 import native as N

    ctx = N.Context(0)
    assert ctx.get_option(N.OPT_AUTOTUNE) == N.AUTOTUNE_OFF
    with pytest.raises(N.OtmError):
        N.check(N.lib().otm_set_option(ctx.handle, N.OPT_AUTOTUNE, 7))
