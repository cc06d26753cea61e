"""torch.autograd wrapper of the log marginal likelihood and its
hand-written adjoint (crava_gpu_loglik_grad).  It exists for the tests:
the backward pass returns the gradients the CUDA kernel computed in the
forward call (the kernel recomputes the per-bin factors itself), so
gradient checks through autograd exercise the same C-ABI entry point a
C++ caller uses."""
from __future__ import annotations

import numpy as np
import torch


class LogMarginal(torch.autograd.Function):
    """L(wavelet_scale [nt], noise_var [nt], wavelet_spec [nzp/2+1, nt, 2])
    on fixed transformed grids of a Context."""

    @staticmethod
    def forward(fctx, scale, noise_var, spec, context, grids):
        sp = spec.detach().cpu().numpy()
        L, gs, gv, gw, _ = context.loglik_grad(*grids, scale.detach().cpu().numpy(),
                                               noise_var.detach().cpu().numpy(), sp)
        dt = scale.dtype
        fctx.save_for_backward(torch.from_numpy(gs).to(dt), torch.from_numpy(gv).to(dt),
                               torch.from_numpy(np.stack([gw.real, gw.imag], -1)).to(dt))
        return torch.tensor(L, dtype=dt)

    @staticmethod
    def backward(fctx, grad_out):
        gs, gv, gw = fctx.saved_tensors
        return grad_out * gs, grad_out * gv, grad_out * gw, None, None


def log_marginal(context, grids, scale, noise_var, spec):
    return LogMarginal.apply(scale, noise_var, spec, context, grids)
