"""Forward-mode (tangent) gradients against reverse mode, on the CPU.

The device differentiates expressions with at most MAX_TANGENT_CONSTS
constants in forward mode (csrc/sr_tangent.cu) and the others in reverse mode
(csrc/sr_adjoint.cu).  Both emulators in tests/emulate.py restate those
kernels' arithmetic over the compiled bytecode; here they run on the same
programs: the gradients must agree to rounding (1e-9 of the constant's
absolute contribution scale in float64, 1e-5 in float32) wherever both are
finite: the forward zero rule (a zero partial gives zero) mirrors the reverse
one (a zero adjoint gives zero) along each constant's single path.  The two
modes multiply the same partials in opposite orders, so an intermediate
product can overflow (or underflow) in one order and not in the other
(forward: pow's 2.4e306 times a division's -5.2e5 before log' brings it
back; reverse: the seed times log' first): such constants, finite in one
mode only, stay below 1% of the population's."""
import numpy as np

from emulate import MAX_TANGENT_CONSTS, adjoint_bytecode, tangent_bytecode
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.evaluator import compile_population
from symbolic_regression_gpu_b200.population import Population


def _dataset(rng, V, N):
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(-3, 3, size=(V, N))
    X[:V, : N // 16] = 0.0  # exact zeros: sqrt'(0), log'(0), flat regions, 0 * inf
    X[V] = X[0] * X[1 % V] + np.sin(X[V - 1]) + 0.1 * rng.standard_normal(N)
    return X


def _compare(pop, X, V, dtype):
    code, offs, _ = compile_population(pop, V)
    co = pop.constant_offsets()
    n_checked = n_mismatch = 0
    with np.errstate(all="ignore"):
        for e in range(pop.num_exprs):
            nc = int(co[e + 1] - co[e])
            if nc == 0 or nc > MAX_TANGENT_CONSTS:
                continue
            prog = code[offs[e]:offs[e + 1]]
            m_r, g_r, a_r = adjoint_bytecode(prog, X, V, nc, dtype=dtype, with_abs=True)
            m_t, g_t, a_t = tangent_bytecode(prog, X, V, nc, dtype=dtype, with_abs=True)
            assert (np.isnan(m_r) and np.isnan(m_t)) or m_r == m_t
            n_mismatch += int(np.sum(np.isfinite(g_r) != np.isfinite(g_t)))
            fin = np.isfinite(g_r) & np.isfinite(g_t) & np.isfinite(a_r)
            err = np.abs(g_r[fin] - g_t[fin]) / np.maximum(a_r[fin], 1e-300)
            tol = 1e-9 if dtype == np.float64 else 1e-5
            assert np.all(err <= tol), (e, err.max())
            n_checked += nc
    assert n_mismatch <= 0.01 * n_checked, (n_mismatch, n_checked)
    return n_checked


def test_tangent_equals_reverse_every_operator_fp64():
    rng = np.random.default_rng(71)
    V, N = 3, 2_000
    X = _dataset(rng, V, N)
    gen = synth.TreeGen(rng, V, p_const=0.3, binary=tuple(range(1, 10)),
                        unary=tuple(range(10, 28)) + (32,))
    exprs = [gen.depth_tree(int(d), full=False) for d in rng.integers(2, 7, 600)]
    assert _compare(Population.from_lists(exprs), X, V, np.float64) > 300


def test_tangent_equals_reverse_protected_workload_fp32():
    w = synth.grad_workload(seed=3, E=200, N=3_000)
    assert _compare(w.population, w.X, w.num_vars, np.float32) > 300
