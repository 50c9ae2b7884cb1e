"""torch.autograd bindings of the EPG derivative kernels.

EPGSignal maps per-atom parameters (T1, T2, B0, B1) and a flip-angle
schedule to the FISP / SR signal on the GPU: the forward pass is
snapmrf_mrf_dict (one B1 block per atom, so every atom uses its own B1), the
backward pass is snapmrf_epg_adjoint.  CRBLoss gives the Cramer-Rao bound
loss of a set of tissues with its flip-angle gradient (snapmrf_crb_gradient).
They serve gradient checks (torch.autograd.gradcheck against central
differences) and schedule design; dictionary generation and matching do not
use them.
"""
from __future__ import annotations

import numpy as np
import torch

from . import api


class EPGSignal(torch.autograd.Function):
    """signal = EPGSignal.apply(params, alpha, schedule, nstates, echo_type)

    params: CUDA float32 [n][4] (T1, T2, B0, B1; B0 is unused by FISP / SR);
    alpha: float32 [T] flip angles in radians (any device);
    schedule: host float32 [4][T] (rows: flip angle, RF phase (must be 0),
    TR, TE; row 0 is replaced by alpha);
    returns CUDA float32 [n][T][2], the complex signal (Re, Im)."""

    @staticmethod
    def forward(ctx, params, alpha, schedule, nstates: int = 101, echo_type: str = "epg_fisp"):
        if not params.is_cuda:
            raise api.SnapMRFError(1, "EPGSignal: params must be a CUDA tensor")
        params = params.detach().to(torch.float32).contiguous()
        n, T = params.shape[0], alpha.shape[0]
        h = np.array(schedule, np.float32, copy=True).reshape(4, -1)[:, :T].copy()
        h[0] = alpha.detach().to("cpu", torch.float32).numpy()
        out = torch.empty((n, T, 2), dtype=torch.float32, device=params.device)
        api.MRF_dict(out, params, h, T, T, n, 1, 4, nstates, echo_type, flags=api.DICT_ALL_B1_BLOCKS)
        ctx.save_for_backward(params)
        ctx.h, ctx.nstates, ctx.echo_type = h, nstates, echo_type
        ctx.alpha_device = alpha.device
        return out

    @staticmethod
    def backward(ctx, grad_out):
        (params,) = ctx.saved_tensors
        n, T = params.shape[0], ctx.h.shape[1]
        g = grad_out.to(torch.float32).contiguous()
        gp = torch.empty((n, 3), dtype=torch.float32, device=params.device)
        ga = torch.empty((T,), dtype=torch.float32, device=params.device)
        api.epg_adjoint(params, ctx.h, T, T, n, g, gp, 4, ctx.nstates, ctx.echo_type, d_grad_alpha=ga)
        grad_params = torch.zeros_like(params)
        grad_params[:, 0] = gp[:, 0]
        grad_params[:, 1] = gp[:, 1]
        grad_params[:, 3] = gp[:, 2]
        return grad_params, ga.to(ctx.alpha_device), None, None, None


class CRBLoss(torch.autograd.Function):
    """loss = CRBLoss.apply(params, alpha, schedule, nstates, echo_type)

    The sum over tissues of the normalised Cramer-Rao bounds of T1 and T2
    (snapmrf_crb_gradient), differentiable in the flip angles: a schedule
    design loop is a torch optimiser over `alpha`.
    params: CUDA float32 [n][4] tissues (T1, T2, B0, B1); alpha: float32 [T]
    flip angles in radians; schedule: host float32 [4][T] (row 0 is replaced
    by alpha, RF phases must be 0); returns a 0-d CUDA tensor."""

    @staticmethod
    def forward(ctx, params, alpha, schedule, nstates: int = 50, echo_type: str = "epg_fisp"):
        params = params.detach().to(torch.float32).contiguous()
        n, T = params.shape[0], alpha.shape[0]
        h = np.array(schedule, np.float32, copy=True).reshape(4, -1)[:, :T].copy()
        h[0] = alpha.detach().to("cpu", torch.float32).numpy()
        loss = torch.empty(n, dtype=torch.float32, device=params.device)
        grad = torch.empty(T, dtype=torch.float32, device=params.device)
        api.crb_gradient(params, h, T, T, n, loss, grad, 4, nstates, echo_type)
        ctx.save_for_backward(grad)
        ctx.alpha_device = alpha.device
        return loss.sum()

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return None, (grad * grad_out).to(ctx.alpha_device), None, None, None
