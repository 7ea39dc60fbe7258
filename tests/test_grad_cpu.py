"""Gradient checks that need no GPU.

* The FP64 gradient oracle (tree reverse mode) against central finite
  differences of the FP64 oracle MSE.
* The compiled bytecode run backwards in FP64 (tests/emulate.py, the
  adjoint kernel's schedule: tape, adjoint spill slots, producer indices)
  against the tree-based oracle gradient.
"""
import numpy as np
import pytest

from emulate import adjoint_bytecode
from oracle import oracle
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.evaluator import compile_population
from symbolic_regression_gpu_b200.population import Population


def _dataset(rng, V, N, lo=-3.0, hi=3.0):
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(lo, hi, size=(V, N))
    X[V] = X[0] * X[1 % V] + np.sin(X[V - 1]) + 0.1 * rng.standard_normal(N)
    return X


def _smooth_population(rng, E, V):
    gen = synth.TreeGen(rng, V, p_const=0.4,
                        unary=(10, 11, 15, 21, 25, 32), binary=(1, 2, 3))
    return Population.from_lists([gen.depth_tree(5, full=False) for _ in range(E)])


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(11)
    V, N = 3, 400
    X = _dataset(rng, V, N)
    pop = _smooth_population(rng, 40, V)
    mse, g = oracle.grad_f64(pop, X)
    cs = pop.values[pop.tokens == 0].astype(np.float32).astype(np.float64)
    co = pop.constant_offsets()
    checked = 0
    for e in range(pop.num_exprs):
        if not np.isfinite(mse[e]):
            continue
        for c in range(co[e], co[e + 1]):
            h = 1e-3 * max(1.0, abs(cs[c]))
            vals = []
            for s in (-2, -1, 1, 2):
                v = cs.copy()
                v[c] += s * h
                # Constants enter the evaluator as float32: use the rounded step.
                v32 = v.astype(np.float32)
                m, _ = oracle.mse_f64(pop.with_constants(v32.astype(np.float64)), X, threads=1)
                vals.append((m[e], float(v32[c]) - cs[c]))
            (m2m, s2m), (m1m, s1m), (m1p, s1p), (m2p, s2p) = vals
            if not all(np.isfinite([m2m, m1m, m1p, m2p])):
                continue
            fd1 = (m1p - m1m) / (s1p - s1m)
            fd2 = (m2p - m2m) / (s2p - s2m)
            # Skip kinks and flat protected regions, where the two stencils disagree.
            if abs(fd1 - fd2) > 1e-3 * max(1.0, abs(fd1)):
                continue
            assert g[c] == pytest.approx(fd1, rel=1e-4, abs=1e-6 * max(1.0, abs(mse[e]))), (e, c)
            checked += 1
    assert checked >= 30


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_bytecode_adjoint_matches_oracle(seed):
    rng = np.random.default_rng(100 + seed)
    V, N = 4, 300
    X = _dataset(rng, V, N)
    gen = synth.TreeGen(rng, V, p_const=0.35, binary=(1, 2, 3, 4, 5, 6, 7, 8, 9),
                        unary=tuple(range(10, 28)) + (32,))
    pop = Population.from_lists([gen.depth_tree(7, full=False) for _ in range(60)]
                                + [gen.sized_tree(61) for _ in range(20)])
    code, offs, _ = compile_population(pop, V)
    mse_o, g_o = oracle.grad_f64(pop, X)
    co = pop.constant_offsets()
    spilled = 0
    for e in range(pop.num_exprs):
        prog = code[offs[e]:offs[e + 1]]
        spilled += int(np.count_nonzero(((prog[:, 0] >> 9) & 7) == 1))
        nc = int(co[e + 1] - co[e])
        mse_b, g_b = adjoint_bytecode(prog, X, V, nc)
        if not np.isfinite(mse_o[e]):
            assert not np.isfinite(mse_b) or mse_b == pytest.approx(mse_o[e])
            continue
        assert mse_b == pytest.approx(mse_o[e], rel=1e-6, abs=1e-12)
        ref = g_o[co[e]:co[e + 1]]
        fin = np.isfinite(ref)
        np.testing.assert_allclose(g_b[fin], ref[fin], rtol=1e-5,
                                   atol=1e-7 * max(1.0, float(np.abs(ref[fin]).max(initial=0))))
        assert np.array_equal(np.isfinite(g_b), fin)
    assert spilled > 0


def test_gradient_of_unreached_constant_is_zero():
    # min(x0, 5 + x1) with x0 in [-3, 3] and x1 in [-3, 3]: 5 + x1 >= 2 > x0
    # only for part of the data; a constant under a protected division by a
    # tiny denominator gets derivative 0 from the protected region.
    rng = np.random.default_rng(3)
    X = _dataset(rng, 2, 256)
    X[0] = -4.0  # min always returns x0
    pop = Population.from_lists([([6, -1, 1, 0, -1], [0, 0, 0, 5.0, 1])])
    _, g = oracle.grad_f64(pop, X)
    assert g[0] == 0.0
