"""torch.autograd binding on the device evaluator.

Tolerances: backward equals the device gradient exactly (same numbers, scaled
by the incoming gradient); gradcheck's central differences of the FP32 forward
pass agree with the analytic gradient to atol 1e-3, rtol 1e-2 at eps 1e-2 on
smooth expressions (FP32 rounding of the MSE divided by the step dominates).
"""
import numpy as np
import pytest
import torch

from symbolic_regression_gpu_b200 import _lib, synth
from symbolic_regression_gpu_b200.autograd import initial_constants, population_mse
from symbolic_regression_gpu_b200.population import Population

pytestmark = pytest.mark.gpu


def _setup(seed, E, N=4096):
    rng = np.random.default_rng(seed)
    V = 2
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(-2, 2, size=(V, N))
    X[V] = np.sin(X[0]) + X[1] * X[0]
    gen = synth.TreeGen(rng, V, p_const=0.5, unary=(10, 11, 15, 21, 25), binary=(1, 2, 3))
    return X, Population.from_lists([gen.depth_tree(4, full=False) for _ in range(E)])


def test_backward_is_device_gradient(evaluator):
    X, pop = _setup(1, 64)
    evaluator.set_data(X)
    c = initial_constants(pop, device="cuda").requires_grad_()
    mse = population_mse(c, evaluator, pop)
    assert mse.device.type == "cuda" and mse.shape == (pop.num_exprs,)
    m_ref, g_ref = evaluator.eval_grad(pop)
    np.testing.assert_array_equal(mse.detach().cpu().numpy(), m_ref)
    w = torch.linspace(0.5, 2.0, pop.num_exprs, device="cuda")
    (mse * w).sum().backward()
    owner = np.repeat(np.arange(pop.num_exprs), np.diff(pop.constant_offsets()))
    np.testing.assert_allclose(c.grad.cpu().numpy(), g_ref * w.cpu().numpy()[owner], rtol=1e-6)


@pytest.mark.parametrize("mode", [_lib.SR_GRAD_CHECKPOINT, _lib.SR_GRAD_RECOMPUTE])
def test_gradcheck_fp32_forward(evaluator, mode):
    X, pop = _setup(2, 6)
    evaluator.set_data(X)
    c = initial_constants(pop, torch.float64).float().double().requires_grad_()
    assert torch.autograd.gradcheck(lambda x: population_mse(x, evaluator, pop, mode), (c,),
                                    eps=1e-2, atol=1e-3, rtol=1e-2)


def test_torch_optimizer_loop(evaluator):
    # A plain torch optimiser over the constants, through the binding.
    w = synth.grad_workload(seed=12, E=64, N=20_000)
    evaluator.set_data(w.X)
    keep = torch.from_numpy(np.isfinite(evaluator.eval_mse(w.population)))
    c = initial_constants(w.population).requires_grad_()
    opt = torch.optim.Adam([c], lr=0.05)
    first = None
    for _ in range(10):
        opt.zero_grad()
        mse = population_mse(c, evaluator, w.population)
        loss = torch.log(mse[keep]).sum()  # every expression's relative fit
        if first is None:
            first = float(loss.detach())
        loss.backward()
        c.grad.nan_to_num_(0.0)
        opt.step()
    assert np.isfinite(float(loss.detach())) and float(loss.detach()) < first
