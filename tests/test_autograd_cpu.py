"""The torch.autograd binding's plumbing, on CPU: a stand-in evaluator backed
by the FP64 gradient oracle runs in double precision, so torch.autograd.gradcheck
(central finite differences) applies with its default tight tolerances."""
import numpy as np
import pytest
import torch

from oracle import oracle
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.autograd import initial_constants, population_mse
from symbolic_regression_gpu_b200.population import Population


class OracleEvaluator:
    """eval_grad through the FP64 oracle, with constants used as given (the
    device evaluator rounds them to float32; the oracle does too, so the
    stand-in evaluates at the float32 constants)."""

    def __init__(self, X):
        self.X = X

    def eval_grad(self, pop, mode=1):
        return oracle.grad_f64(pop, self.X, threads=2)


def _setup(seed=3, E=6):
    rng = np.random.default_rng(seed)
    V, N = 2, 200
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(-2, 2, size=(V, N))
    X[V] = np.sin(X[0]) + X[1] * X[0]
    gen = synth.TreeGen(rng, V, p_const=0.5, unary=(10, 11, 15, 21, 25), binary=(1, 2, 3))
    pop = Population.from_lists([gen.depth_tree(4, full=False) for _ in range(E)])
    return X, pop


def test_forward_values_and_owner_mapping():
    X, pop = _setup()
    ev = OracleEvaluator(X)
    c = initial_constants(pop, torch.float64).requires_grad_()
    mse = population_mse(c, ev, pop)
    ref, g = oracle.grad_f64(pop, X)
    np.testing.assert_allclose(mse.detach().numpy(), ref)
    w = torch.arange(1, pop.num_exprs + 1, dtype=torch.float64)
    (mse * w).sum().backward()
    owner = np.repeat(np.arange(pop.num_exprs), np.diff(pop.constant_offsets()))
    np.testing.assert_allclose(c.grad.numpy(), g * (owner + 1))


def test_gradcheck_against_finite_differences():
    X, pop = _setup(seed=5, E=4)
    ev = OracleEvaluator(X)
    # The evaluator reads constants as float32; gradcheck perturbs in float64,
    # so start from float32-representable values and use a step that survives
    # the rounding.
    c = initial_constants(pop, torch.float64)
    c = c.float().double().requires_grad_()
    if c.numel() == 0:
        pytest.skip("no constants")
    assert torch.autograd.gradcheck(lambda x: population_mse(x, ev, pop), (c,),
                                    eps=1e-3, atol=1e-4, rtol=1e-3)


def test_wrong_constant_count_is_rejected():
    X, pop = _setup()
    ev = OracleEvaluator(X)
    with pytest.raises(ValueError):
        population_mse(torch.zeros(1000, dtype=torch.float64), ev, pop)
