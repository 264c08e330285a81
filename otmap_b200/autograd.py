"""torch.autograd binding of the GPU solver and its implicit adjoint.

    fwd = transport_map(density_cells, n)          # (V, 2) forward mesh, differentiable

Forward: otm_solve on the density (float64 CUDA tensor in face order). Backward:
otm_adjoint with dL/dfwd, returning dL/ddensity. Only the density and the final map
are kept for the backward pass. PyTorch is the harness here; the computation runs in
the CUDA library.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import native as N


class _TransportMap(torch.autograd.Function):
    @staticmethod
    def forward(ctx, density, n, threshold, max_iter, adjoint_mode, adjoint_tol, context):
        if not density.is_cuda or density.dtype != torch.float64:
            raise TypeError("density must be a float64 CUDA tensor")
        d = density.contiguous()
        fwd = torch.empty(((n + 1) ** 2, 2), dtype=torch.float64, device=d.device)
        opt = N.default_options()
        opt.threshold = threshold
        opt.max_iter = max_iter
        st = N.SolveStatsC()
        torch.cuda.current_stream(d.device).synchronize()
        N.check(N.lib().otm_solve(context.handle, n, C.c_void_p(d.data_ptr()), C.byref(opt),
                                  C.c_void_p(fwd.data_ptr()), None, C.byref(st)))
        ctx.save_for_backward(d, fwd)
        ctx.n = n
        ctx.mode = adjoint_mode
        ctx.tol = adjoint_tol
        ctx.context = context
        ctx.stats = st
        return fwd

    @staticmethod
    def backward(ctx, grad_fwd):
        d, fwd = ctx.saved_tensors
        g = grad_fwd.contiguous().to(torch.float64)
        out = torch.empty_like(d)
        opt = N.AdjointOptionsC()
        N.lib().otm_default_adjoint_options(C.byref(opt))
        opt.mode = ctx.mode
        opt.tol = ctx.tol
        st = N.AdjointStatsC()
        torch.cuda.current_stream(d.device).synchronize()
        N.check(N.lib().otm_adjoint(ctx.context.handle, ctx.n, C.c_void_p(d.data_ptr()), C.c_void_p(fwd.data_ptr()),
                                    C.c_void_p(g.data_ptr()), C.byref(opt), C.c_void_p(out.data_ptr()),
                                    C.byref(st)))
        ctx.context.last_adjoint_stats = st
        return out, None, None, None, None, None, None


def transport_map(density, n, threshold=1e-7, max_iter=1000, adjoint="krylov", adjoint_tol=1e-10, context=None):
    """Forward mesh of the transport map of `density` (float64 CUDA tensor, N cells),
    differentiable with respect to the density through the implicit adjoint.
    adjoint: "krylov" (converged) or "one_step" (one Poisson solve)."""
    mode = N.ADJOINT_KRYLOV if adjoint == "krylov" else N.ADJOINT_ONE_STEP
    ctx = context or N.default_context()
    return _TransportMap.apply(density, int(n), float(threshold), int(max_iter), mode, float(adjoint_tol), ctx)


def blur_torch(img, sigma):
    """Separable Gaussian blur (radius ceil(3 sigma), mirror borders including the edge
    sample), differentiable; matches otmap_b200.workloads.gaussian_blur."""
    import math

    if sigma <= 0:
        return img
    r = max(1, int(math.ceil(3.0 * sigma)))
    t = torch.arange(-r, r + 1, dtype=img.dtype, device=img.device)
    k = torch.exp(-0.5 * (t / sigma) ** 2)
    k = k / k.sum()
    out = img
    for dim in (0, 1):
        n = out.shape[dim]
        idx = torch.arange(-r, n + r, device=img.device)
        idx = torch.where(idx < 0, -idx - 1, idx)
        idx = torch.where(idx >= n, 2 * n - 1 - idx, idx)
        p = out.index_select(dim, idx)
        acc = torch.zeros_like(out)
        for q in range(2 * r + 1):
            acc = acc + k[q] * p.narrow(dim, q, n)
        out = acc
    return out


class _BarycenterLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, densities, weights, target, res, threshold, max_iter, adjoint_mode, adjoint_tol, context):
        if not densities.is_cuda or densities.dtype != torch.float64 or densities.dim() != 2:
            raise TypeError("densities must be a (count, n*n) float64 CUDA tensor")
        count, cells = densities.shape
        n = int(round(cells ** 0.5))
        d = densities.contiguous()
        t = target.contiguous().to(device=d.device, dtype=torch.float64)
        grads = torch.empty_like(d)
        image = torch.empty((res, res), dtype=torch.float64, device=d.device)
        opt = N.default_options()
        opt.threshold = threshold
        opt.max_iter = max_iter
        aopt = N.AdjointOptionsC()
        N.lib().otm_default_adjoint_options(C.byref(aopt))
        aopt.mode = adjoint_mode
        aopt.tol = adjoint_tol
        st = N.BarycenterStatsC()
        loss = C.c_double(0.0)
        dp = (C.c_void_p * count)(*[d[k].data_ptr() for k in range(count)])
        gp = (C.c_void_p * count)(*[grads[k].data_ptr() for k in range(count)])
        w = (C.c_double * count)(*[float(x) for x in weights])
        torch.cuda.current_stream(d.device).synchronize()
        N.check(N.lib().otm_barycenter_loss(context.handle, n, count, dp, w, res, C.c_void_p(t.data_ptr()),
                                            C.byref(opt), C.byref(aopt), C.c_void_p(image.data_ptr()),
                                            C.byref(loss), gp, C.byref(st)))
        ctx.save_for_backward(grads)
        context.last_barycenter_stats = st
        context.last_barycenter_image = image
        return torch.tensor(loss.value, dtype=torch.float64, device=d.device)

    @staticmethod
    def backward(ctx, grad_loss):
        (grads,) = ctx.saved_tensors
        return grad_loss * grads, None, None, None, None, None, None, None, None


def barycenter_loss(densities, weights, target, res=None, threshold=1e-7, max_iter=1000, adjoint="krylov",
                    adjoint_tol=1e-10, context=None):
    """L = sum (barycenter image - target)^2 of the barycenters pipeline for densities (a
    (count, n*n) float64 CUDA tensor, face order), differentiable with respect to them. The
    gradient is computed with the forward pass (one library call) and kept until backward;
    the image of the forward pass is left in context.last_barycenter_image."""
    mode = N.ADJOINT_KRYLOV if adjoint == "krylov" else N.ADJOINT_ONE_STEP
    ctx = context or N.default_context()
    res = int(res or target.shape[0])
    return _BarycenterLoss.apply(densities, tuple(float(x) for x in weights), target, res, float(threshold),
                                 int(max_iter), mode, float(adjoint_tol), ctx)
