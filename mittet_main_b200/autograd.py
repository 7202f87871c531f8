"""The FWI misfit as a differentiable PyTorch function.

forward(sigma) runs the batched forward solve and the discrete adjoint on the
GPU (mittet_gradient: checkpointed forward, recomputation, adjoint sweep) and
returns the misfit 0.5 sum |S - obs|^2 over shots, receivers and frequencies;
backward multiplies the stored gradient d(misfit)/d(sigma) (satan_i layout:
[nz, ny, nx], zero in the CPML frame) by the incoming gradient.  A CUDA sigma
goes to the solver from device memory (mittet_set_model_device), without a
host round trip.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import MittetSolver


class MisfitFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma: torch.Tensor, solver: MittetSolver, obs: np.ndarray, nt: int,
                checkpoint_every: int = 200):
        if sigma.is_cuda:
            solver.set_model_device(sigma.detach().to(torch.float64).contiguous())
        else:
            solver.set_model(sigma.detach().to(torch.float64).numpy())
        misfit, grad = solver.gradient(nt, obs, checkpoint_every)
        ctx.save_for_backward(torch.from_numpy(grad).to(device=sigma.device, dtype=sigma.dtype))
        return sigma.new_tensor(misfit)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None, None, None, None


def fwi_misfit(sigma: torch.Tensor, solver: MittetSolver, obs: np.ndarray, nt: int,
               checkpoint_every: int = 200) -> torch.Tensor:
    """Differentiable misfit of conductivity ``sigma`` ([nz, ny, nx])."""
    return MisfitFunction.apply(sigma, solver, obs, nt, checkpoint_every)
