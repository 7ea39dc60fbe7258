"""The condition-aware parity rule (oracle.error_bound, oracle/sr_oracle.c
sro_error_bound) tested on the CPU, before the GPU tests rely on it.

The rule: every datapoint must lie within max(4 ulp, its running forward
error bound) of the reference's value unless it is flagged (a discontinuity,
singularity or overflow within its bound); every expression without a flagged
datapoint must lie within max(1e-6, its bound) of the reference's MSE.  The
bound is built from the documented maximum errors of the two implementations'
functions, so (1) it must cover an evaluator whose transcendental results
differ from glibc's by up to the device's documented ulps, and (2) it must not
cover a planted operator mistake.  Both are checked here with a perturbed
evaluator of the float path (oracle.predict_f32_perturbed)."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle
from symbolic_regression_gpu_b200 import opcodes as op
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.population import Population


def _populations():
    rng = np.random.default_rng(9)
    X = rng.uniform(-4, 4, size=(4, 2000)).astype(np.float32)
    allops = synth.small_random_population(9, 250, 3, max_len=40, binary=list(op.BINARY_OPS),
                                           unary=list(op.UNARY_OPS))
    p = synth.plain_workload(seed=7, E=250, N=2000)
    b = synth.batched_workload(seed=8, E=250, N=2000, generations=2)
    g = synth.grad_workload(seed=10, E=200, N=2000)
    return [("all operators", allops, X), ("plain", p.population, p.X),
            ("batched", b.population, b.X), ("constants", g.population, g.X)]


@pytest.mark.parametrize("case", range(4))
def test_bound_covers_the_documented_differences(case):
    name, pop, X = _populations()[case]
    bnd = oracle.error_bound(pop, X, mode=0, per_datapoint=True, threads=4)
    ref = oracle.predict_f32(pop, X, threads=4)
    # The bound's centre is the reference's own float evaluation.
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(bnd["pred"]), fin)
    assert (bnd["pred"][fin].astype(np.float32) == ref[fin]).all()
    ref_mse = oracle.mse_f32(pop, X, threads=4)
    for seed in range(3):
        got = oracle.predict_f32_perturbed(pop, X, oracle.DEVICE_ULPS, seed=seed)
        r = oracle.datapoint_parity(got, ref, bnd["bound"], bnd["flag"])
        assert r["violations"] == 0, (name, seed, r)
        assert r["max_excess_over_allowance"] <= 1.0
        m = oracle.mse_of_predictions(got, X[-1])
        rm = oracle.mse_parity(m, ref_mse, bnd["mse_bound"], bnd["flagged"])
        assert rm["violations"] == 0, (name, seed, rm)
    print(name, r, rm)


def test_bound_does_not_cover_a_planted_operator_mistake():
    """sin and cos swapped in one evaluator: the rule must fail."""
    p = synth.plain_workload(seed=7, E=250, N=2000)
    bnd = oracle.error_bound(p.population, p.X, mode=0, per_datapoint=True, threads=4)
    ref = oracle.predict_f32(p.population, p.X, threads=4)
    bad = oracle.predict_f32_perturbed(p.population, p.X, oracle.DEVICE_ULPS, seed=1,
                                       swap_sin_cos=True)
    r = oracle.datapoint_parity(bad, ref, bnd["bound"], bnd["flag"])
    assert r["violations"] > 1000, r
    m = oracle.mse_of_predictions(bad, p.X[-1])
    rm = oracle.mse_parity(m, oracle.mse_f32(p.population, p.X), bnd["mse_bound"],
                           bnd["flagged"])
    assert rm["violations"] > 10, rm


def test_bound_is_zero_for_ieee_only_expressions():
    """With IEEE operators only both evaluations are bit-identical: the
    bound is 0 at every datapoint, so the rule demands bit equality."""
    rng = np.random.default_rng(3)
    X = rng.uniform(-3, 3, size=(4, 500)).astype(np.float32)
    pop = synth.small_random_population(3, 80, 3, max_len=31,
                                        binary=(op.ADD, op.SUB, op.MUL, op.LOOSE_DIV),
                                        unary=(op.NEG, op.ABS, op.LOOSE_SQRT))
    bnd = oracle.error_bound(pop, X, mode=0, per_datapoint=True)
    assert (bnd["bound"] == 0).all()
    assert (bnd["mse_bound"] == 0).all()


def test_flags_mark_the_discontinuities():
    """A protected division whose divisor's bound reaches the 1e-9 boundary
    and an exp that may or may not overflow are flagged; exact operands and
    results C99 fixes exactly (sin(0) = 0) are not."""
    C, V = op.TOK_CONST, op.TOK_VAR
    # 88.72283935546875: the float just above ln(FLT_MAX) (e^x is 2.5 ulps
    # past FLT_MAX: inf correctly rounded, FLT_MAX within 2 ulps of error).
    X = np.array([[1e-9, 0.5, 88.7228394, 0.0], [0.0, 0.0, 0.0, 0.0]], np.float32)
    pop = Population.from_lists([
        ([op.LOOSE_DIV, C, V], [0.0, 1.0, 0.0]),                # exact divisor
        ([op.LOOSE_DIV, C, op.SIN, op.SUB, V, V], [0, 1.0, 0, 0, 0, 0]),  # sin(0) = 0 exactly
        ([op.LOOSE_DIV, C, op.SIN, V], [0, 1.0, 0, 0]),         # sin(1e-9) at the boundary
        ([op.EXP, V], [0.0, 0.0]),                              # e^x near FLT_MAX
    ])
    bnd = oracle.error_bound(pop, X, mode=0, per_datapoint=True)
    f = bnd["flag"]
    assert not f[0].any() and not f[1].any()
    assert f[2, 0] and not f[2, 1:].any()
    assert f[3, 2] and not f[3, [0, 1, 3]].any()


def test_fp64_mode_centre_is_the_fp64_evaluation():
    w = synth.plain_workload(seed=5, E=120, N=3000)
    bnd = oracle.error_bound(w.population, w.X, mode=1)
    m64, cnt = oracle.mse_f64(w.population, w.X)
    assert np.array_equal(cnt, bnd["valid"])
    ok = np.isfinite(m64)
    assert np.allclose(bnd["mse"][ok], m64[ok], rtol=1e-12, atol=0)


def test_golden_predictions_within_the_rule_of_themselves():
    """Sanity: the reference's golden predictions satisfy the rule against
    themselves with no flag needed (zero differences)."""
    pop, d = load_golden("eval_all_ops.npz")
    bnd = oracle.error_bound(pop, d["X"], mode=0, per_datapoint=True)
    fin = np.isfinite(d["pred"])
    assert (bnd["pred"][fin].astype(np.float32) == d["pred"][fin]).all()
    r = oracle.datapoint_parity(d["pred"], d["pred"], bnd["bound"], bnd["flag"])
    assert r["violations"] == 0
