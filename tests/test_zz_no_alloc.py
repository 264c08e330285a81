"""The allocation-free solve (otm_solve_noalloc) against otm_solve, through the C ABI.

otm_solve_noalloc is for callers that cannot let a library call cudaMalloc: a host
whose allocator reserved all device memory at start-up, or a process under a hard
device-memory budget. Its working memory is one fixed static device array shared by
every call, and it runs the dense-product Poisson solve, so it matches otm_solve to the
solver tolerance (same iterations, positions within 1e-6), not bit for bit. These tests
check that two calls in a row -- the second one starting from the first one's leftovers
in that array -- reproduce otm_solve, that a warmed-up call leaves the device's free
memory unchanged, that sizes below one transform tile, odd sizes and the largest
allowed size work, and that sizes past the array's limit are refused. Collected last so
that a failure here does not stop the rest of the suite; passes both alone and after
the other tests.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POS_TOL = 1e-6  # vertex positions, as in the other parity tests


def _solve_ref(N, ctx, n, dens):
    fwd = np.empty(((n + 1) ** 2, 2))
    adj = np.empty(n * n)
    st = N.SolveStatsC()
    N.check(N.lib().otm_solve(ctx.handle, n, N.ptr(dens), None, N.ptr(fwd), N.ptr(adj), C.byref(st)))
    return fwd, adj, st


def test_noalloc_two_calls_match_solve():
    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    ctx = N.Context(0)
    L = N.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(64, W.to_cells(W.gaussian_mixture(64, 11))), (64, W.to_cells(W.blurred_shapes(64, 12, sigma_px=1.5))),
             (256, W.to_cells(W.gaussian_mixture(256, 13)))]
    for n, dens in cases:
        fwd_ref, adj_ref, st_ref = _solve_ref(N, ctx, n, dens)
        # first call: device buffers; second call: host buffers (same density)
        d_in = torch.from_numpy(dens).cuda()
        d_fwd = torch.full(((n + 1) ** 2, 2), float("nan"), dtype=torch.float64, device="cuda")
        d_adj = torch.empty(n * n, dtype=torch.float64, device="cuda")
        st1 = N.SolveStatsC()
        torch.cuda.synchronize()
        N.check(L.otm_solve_noalloc(n, C.c_void_p(d_in.data_ptr()), None, C.c_void_p(d_fwd.data_ptr()),
                                    C.c_void_p(d_adj.data_ptr()), C.byref(st1), C.c_void_p(stream)))
        fwd1 = d_fwd.cpu().numpy()
        h_fwd = np.full(((n + 1) ** 2, 2), np.nan)
        h_adj = np.empty(n * n)
        st2 = N.SolveStatsC()
        N.check(L.otm_solve_noalloc(n, N.ptr(dens), None, N.ptr(h_fwd), N.ptr(h_adj), C.byref(st2),
                                    C.c_void_p(stream)))
        for fwd, adj, st in ((fwd1, d_adj.cpu().numpy(), st1), (h_fwd, h_adj, st2)):
            assert st.iterations == st_ref.iterations
            assert st.outcome == st_ref.outcome
            assert np.abs(fwd - fwd_ref).max() <= POS_TOL
            np.testing.assert_allclose(adj, adj_ref, rtol=1e-13, atol=0)
            np.testing.assert_allclose(st.residual, st_ref.residual, rtol=1e-6, atol=1e-14)
    ctx.close()


def test_noalloc_rejects_sizes_past_its_limit():
    from otmap_b200 import native as N

    L = N.lib()
    n = 257
    dens = np.ones(n * n)
    fwd = np.empty(((n + 1) ** 2, 2))
    rc = L.otm_solve_noalloc(n, N.ptr(dens), None, N.ptr(fwd), None, None, None)
    assert rc == N.ERR_BAD_ARG
    assert b"256" in L.otm_last_error()


def _noalloc(N, n, dens, stream):
    fwd = np.full(((n + 1) ** 2, 2), np.nan)
    adj = np.empty(n * n)
    st = N.SolveStatsC()
    N.check(N.lib().otm_solve_noalloc(n, N.ptr(dens), None, N.ptr(fwd), N.ptr(adj), C.byref(st), C.c_void_p(stream)))
    return fwd, adj, st


@pytest.mark.parametrize("n", [1, 37, 255])
def test_noalloc_odd_and_edge_sizes_match_solve(n):
    """n = 1 (nothing to solve), 37 (odd, smaller than one 64-wide transform tile) and
    255 (the largest odd size, 256 stencil tiles) against otm_solve, twice in a row."""
    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    ctx = N.Context(0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    dens = W.to_cells(W.gaussian_mixture(n, 21 + n)) if n > 1 else np.ones(1)
    fwd_ref, adj_ref, st_ref = _solve_ref(N, ctx, n, dens)
    for _ in range(2):
        fwd, adj, st = _noalloc(N, n, dens, stream)
        assert st.iterations == st_ref.iterations
        assert st.outcome == st_ref.outcome
        assert np.abs(fwd - fwd_ref).max() <= POS_TOL
        np.testing.assert_allclose(adj, adj_ref, rtol=1e-13, atol=0)
    ctx.close()


def test_noalloc_leaves_free_device_memory_unchanged():
    """After a first call on the device (which loads the kernels and runs the one-time
    check), further calls change the device's free memory by nothing."""
    import torch

    from otmap_b200 import native as N
    from otmap_b200 import workloads as W

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    n = 128
    dens = W.to_cells(W.gaussian_mixture(n, 5))
    _noalloc(N, n, dens, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for seed in (6, 7):
        _noalloc(N, n, W.to_cells(W.gaussian_mixture(n, seed)), stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
