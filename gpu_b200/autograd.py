"""torch.autograd wrappers of the projector and its matched adjoint.

``ForwardProject.apply(vol, geom, views)`` returns A x for a range of views
and backpropagates with the exact adjoint Aᵀ (``ctr_backproject``), so the
gradient of any loss of A x is the engine's matched adjoint applied to the
upstream gradient.  ``BackProject`` is the transpose pair.

``data_fidelity_loss`` evaluates 0.5 ||A x - b||² in chunks of views: the
forward chunk's projections are dropped after the residual is reduced, and the
backward pass recomputes A x chunk by chunk (per-view-chunk recomputation),
so large sinograms never hold an A x-sized intermediate.  ``tv_iso`` is the
isotropic TV of the reference's TV_norm_kernel (V63/kernel_tool_functions.cu:
39-65) written in torch for its gradient.
"""
from __future__ import annotations

import torch

from . import ctrecon


def _check(vol):
    if not vol.is_cuda or vol.dtype != torch.float32 or not vol.is_contiguous():
        raise TypeError("volume must be a contiguous float32 CUDA tensor")


class ForwardProject(torch.autograd.Function):
    """y = A x over views [v0, v0 + n); dy -> Aᵀ dy."""

    @staticmethod
    def forward(ctx, vol, geom, v0=0, n=None):
        _check(vol)
        n = geom.n_views - v0 if n is None else n
        out = torch.empty((n,) + geom.view_shape, device=vol.device, dtype=torch.float32)
        geom.forward(vol, out, v0, n)
        ctx.geom, ctx.v0, ctx.n = geom, v0, n
        return out

    @staticmethod
    def backward(ctx, gy):
        g = ctx.geom
        gx = torch.empty(g.vol_shape, device=gy.device, dtype=torch.float32)
        g.backproject(gy.contiguous().float(), gx, ctx.v0, ctx.n)
        return gx, None, None, None


class BackProject(torch.autograd.Function):
    """x = Aᵀ y over views [v0, v0 + n); dx -> A dx."""

    @staticmethod
    def forward(ctx, sino, geom, v0=0, n=None):
        n = geom.n_views - v0 if n is None else n
        out = torch.empty(geom.vol_shape, device=sino.device, dtype=torch.float32)
        geom.backproject(sino.contiguous().float(), out, v0, n)
        ctx.geom, ctx.v0, ctx.n = geom, v0, n
        return out

    @staticmethod
    def backward(ctx, gx):
        g = ctx.geom
        gy = torch.empty((ctx.n,) + g.view_shape, device=gx.device, dtype=torch.float32)
        g.forward(gx.contiguous().float(), gy, ctx.v0, ctx.n)
        return gy, None, None, None


class _ChunkedFidelity(torch.autograd.Function):
    """0.5 ||A x - b||² with per-view-chunk recomputation in backward."""

    @staticmethod
    def forward(ctx, vol, b, geom, chunk):
        _check(vol)
        total = torch.zeros((), device=vol.device, dtype=torch.float64)
        buf = torch.empty((min(chunk, geom.n_views),) + geom.view_shape, device=vol.device, dtype=torch.float32)
        for v0 in range(0, geom.n_views, chunk):
            n = min(chunk, geom.n_views - v0)
            ax = buf[:n]
            geom.forward(vol, ax, v0, n)
            r = ax - b[v0:v0 + n]
            total += 0.5 * torch.sum(r.double() * r.double())
        ctx.save_for_backward(vol, b)
        ctx.geom, ctx.chunk = geom, chunk
        return total

    @staticmethod
    def backward(ctx, gtotal):
        """d/dx = A^T (A x - b) and d/db = -(A x - b), each scaled by the
        incoming gradient; A x is recomputed chunk by chunk."""
        vol, b = ctx.saved_tensors
        g, chunk = ctx.geom, ctx.chunk
        want_x, want_b = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        grad = torch.zeros(g.vol_shape, device=vol.device, dtype=torch.float32) if want_x else None
        grad_b = torch.empty_like(b, dtype=torch.float32) if want_b else None
        buf = torch.empty((min(chunk, g.n_views),) + g.view_shape, device=vol.device, dtype=torch.float32)
        for v0 in range(0, g.n_views, chunk):
            n = min(chunk, g.n_views - v0)
            ax = buf[:n]
            g.forward(vol, ax, v0, n)                  # recompute this chunk
            r = (ax - b[v0:v0 + n]).contiguous()
            if want_x:
                g.backproject(r, grad, v0, n, flags=ctrecon.BP_ACCUMULATE)
            if want_b:
                grad_b[v0:v0 + n] = -r
        gs = gtotal.float()
        return (grad * gs if want_x else None), (grad_b.to(b.dtype) * gs if want_b else None), None, None


def data_fidelity_loss(vol, b, geom, chunk=64):
    """0.5 ||A x - b||² (FP64 scalar), gradient Aᵀ(A x - b), recomputed in view chunks."""
    return _ChunkedFidelity.apply(vol, b, geom, chunk)


def tv_iso(vol):
    """Isotropic forward-difference TV with the reference's boundary cases
    (V63/kernel_tool_functions.cu:39-65): at the last x/y/z plane the missing
    difference is left out; the corner voxel contributes 0."""
    d = vol
    dx = torch.zeros_like(d)
    dy = torch.zeros_like(d)
    dz = torch.zeros_like(d)
    dx[:, :, :-1] = d[:, :, :-1] - d[:, :, 1:]
    dy[:, :-1, :] = d[:, :-1, :] - d[:, 1:, :]
    dz[:-1, :, :] = d[:-1, :, :] - d[1:, :, :]
    sq = dx * dx + dy * dy + dz * dz
    # sqrt(x^2) at single-difference boundaries is |x|; the offset keeps the
    # gradient finite where all differences vanish; terms in float, sum in FP64
    return torch.sum((torch.sqrt(sq + 1e-20) - (sq == 0).to(d.dtype) * 1e-10).double())


def recon_loss(vol, b, geom, lam, chunk=64):
    """0.5 ||A x - b||² + lam * TV_iso(x)."""
    return data_fidelity_loss(vol, b, geom, chunk) + lam * tv_iso(vol)
