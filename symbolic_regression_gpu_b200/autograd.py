"""torch.autograd binding of the fused forward + adjoint.

``population_mse(constants, evaluator, population)`` returns the MSE of every
expression of ``population`` (float [E]) with the population's constants
replaced by ``constants`` (float [C], token order, CSR over expressions as
sr_count_constants numbers them), and is differentiable in ``constants``:
the backward pass is d loss / d c_k = d loss / d mse_e(k) * d mse_e(k) / d c_k
with the per-constant derivatives from sr_eval_grad (no reference
counterpart: the reference evaluates MSE only).

The evaluator computes in FP32 whatever the tensor dtype; a float64 input
gives float64 outputs holding FP32-accurate values.  Tensors may live on any
device: the library reads host buffers, so inputs are copied to the host and
results copied back to the input's device.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .population import Population


def _const_owner(pop: Population) -> np.ndarray:
    """Expression index of every constant (token order)."""
    co = pop.constant_offsets()
    return np.repeat(np.arange(pop.num_exprs, dtype=np.int64), np.diff(co))


class PopulationMSE(torch.autograd.Function):
    """MSE [E] of a population as a function of its constants [C]."""

    @staticmethod
    def forward(ctx, constants: torch.Tensor, evaluator, population: Population,
                mode: int = _lib.SR_GRAD_CHECKPOINT):
        if constants.dim() != 1:
            raise ValueError("constants must be a 1-D tensor")
        n = int(np.count_nonzero(population.tokens == 0))
        if constants.numel() != n:
            raise ValueError(f"population has {n} constants, got {constants.numel()}")
        c = constants.detach().to("cpu", torch.float64).numpy()
        pop = population.with_constants(c)
        mse, grad = evaluator.eval_grad(pop, mode=mode)
        owner = torch.from_numpy(_const_owner(population)).to(constants.device)
        ctx.save_for_backward(torch.from_numpy(grad).to(constants.device, constants.dtype), owner)
        return torch.from_numpy(mse).to(constants.device, constants.dtype)

    @staticmethod
    def backward(ctx, grad_mse: torch.Tensor):
        grad, owner = ctx.saved_tensors
        g = None
        if ctx.needs_input_grad[0]:
            g = grad_mse.index_select(0, owner) * grad
        return g, None, None, None


def population_mse(constants: torch.Tensor, evaluator, population: Population,
                   mode: int = _lib.SR_GRAD_CHECKPOINT) -> torch.Tensor:
    return PopulationMSE.apply(constants, evaluator, population, mode)


def initial_constants(population: Population, dtype=torch.float32, device=None) -> torch.Tensor:
    """The population's own constants as a tensor (token order)."""
    c = population.values[population.tokens == 0]
    return torch.tensor(c, dtype=dtype, device=device)
