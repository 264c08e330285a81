"""The bounded device-side waits of the row transforms (a bulk copy completing on an
mbarrier). With OTM_OPT_WAIT_TEST the waits expect bytes that never arrive and give up
after about 1 ms: the instance is flagged, the call returns OTM_ERR_TIMEOUT, and the
context stays usable -- the next solve is identical to one that never saw the fault.
No GPU fault, trap or hang is involved: the wait simply runs out."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_the_context_recovers():
    from otmap_b200 import native as N
    from otmap_b200 import otmap as ot
    from otmap_b200 import workloads as W

    ctx = N.Context(0)
    n = 64
    d = W.to_cells(W.gaussian_mixture(n, 5))
    s = ot.GridBasedTransportSolver(ctx)
    s.set_verbose_level(0)
    s.init(n)
    good = s.solve(d)

    N.check(N.lib().otm_set_option(ctx.handle, N.OPT_WAIT_TEST, 1))
    for loop in (N.LOOP_GRAPH, N.LOOP_HOST):
        ctx.set_loop(loop)
        with pytest.raises(N.OtmError) as e:
            s.solve(d)
        assert e.value.code == N.ERR_TIMEOUT
    batch = [W.gaussian_mixture(k, 9) for k in (64, 128)]
    with pytest.raises(N.OtmError) as e:
        ot.solve_batch(batch, context=ctx)
    assert e.value.code == N.ERR_TIMEOUT

    ctx.set_loop(N.LOOP_GRAPH)
    N.check(N.lib().otm_set_option(ctx.handle, N.OPT_WAIT_TEST, 0))
    again = s.solve(d)
    assert again.stats.iterations == good.stats.iterations
    assert np.array_equal(again.fwd_mesh(), good.fwd_mesh())
    maps = ot.solve_batch(batch, context=ctx)
    assert all(m.stats.outcome == N.CONVERGED for m in maps)
    ctx.close()


def test_tensor_transform_wait_runs_out_and_the_context_recovers():
    """The tensor-core transform's stage barriers (TMA transaction counts): under
    OTM_OPT_WAIT_TEST they expect 16 bytes more than the copies bring, every wait gives up
    after about 1 ms with the copies landed, the instance is flagged and the call returns
    OTM_ERR_TIMEOUT; afterwards the same context solves as before."""
    from otmap_b200 import native as N
    from otmap_b200 import otmap as ot
    from otmap_b200 import workloads as W

    ctx = N.Context(0)
    ctx.set_precision(N.PRECISION_SPLIT)
    ctx.set_poisson(N.POISSON_TENSOR)
    n = 256
    d = W.to_cells(W.gaussian_mixture(n, 5))
    s = ot.GridBasedTransportSolver(ctx)
    s.set_verbose_level(0)
    s.init(n)
    good = s.solve(d)
    N.check(N.lib().otm_set_option(ctx.handle, N.OPT_WAIT_TEST, 1))
    with pytest.raises(N.OtmError) as e:
        s.solve(d)
    assert e.value.code == N.ERR_TIMEOUT
    N.check(N.lib().otm_set_option(ctx.handle, N.OPT_WAIT_TEST, 0))
    again = s.solve(d)
    assert again.stats.iterations == good.stats.iterations
    assert np.array_equal(again.fwd_mesh(), good.fwd_mesh())
    ctx.close()


@pytest.mark.parametrize("loop", ["graph", "host"])
def test_adjoint_wait_runs_out_and_the_context_recovers(loop):
    """The adjoint's Poisson solves use the same row transforms: under OTM_OPT_WAIT_TEST the
    Krylov adjoint (its Arnoldi cycles as a graph launch, or step by step in the host loop)
    returns OTM_ERR_TIMEOUT after a bounded number of steps; with the option off, the same
    context's next adjoint equals that of a context that never saw the fault."""
    import ctypes as C

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    n = 64
    d = W.to_cells(W.gaussian_mixture(n, 7))
    q = np.random.default_rng(3).standard_normal(((n + 1) ** 2, 2))

    def adjoint(ctx, fwd):
        g = np.empty(n * n)
        opt = N.AdjointOptionsC()
        N.lib().otm_default_adjoint_options(C.byref(opt))
        opt.mode = N.ADJOINT_KRYLOV
        opt.max_iter = 60
        st = N.AdjointStatsC()
        N.check(N.lib().otm_adjoint(ctx.handle, n, N.ptr(d), N.ptr(fwd), N.ptr(q), C.byref(opt), N.ptr(g),
                                    C.byref(st)))
        return g

    def forward(ctx):
        fwd = np.empty(((n + 1) ** 2, 2))
        opt = N.default_options()
        opt.threshold = 1e-13
        opt.max_iter = 300
        st = N.SolveStatsC()
        N.check(N.lib().otm_solve(ctx.handle, n, N.ptr(d), C.byref(opt), N.ptr(fwd), None, C.byref(st)))
        return fwd

    clean = N.Context(0)
    fwd = forward(clean)
    good = adjoint(clean, fwd)
    clean.close()

    ctx = N.Context(0)
    ctx.set_loop(N.LOOP_GRAPH if loop == "graph" else N.LOOP_HOST)
    adjoint(ctx, fwd)  # workspace and step graph built before the fault
    N.check(N.lib().otm_set_option(ctx.handle, N.OPT_WAIT_TEST, 1))
    with pytest.raises(N.OtmError) as e:
        adjoint(ctx, fwd)
    assert e.value.code == N.ERR_TIMEOUT
    N.check(N.lib().otm_set_option(ctx.handle, N.OPT_WAIT_TEST, 0))
    again = adjoint(ctx, fwd)
    assert np.array_equal(again, good)
    ctx.close()
