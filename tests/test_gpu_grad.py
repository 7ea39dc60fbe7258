"""Forward + adjoint kernel against the FP64 gradient oracle and the FP32
bytecode emulator.

The device computes forward values, local partials and adjoint products in
FP32 and accumulates each constant's gradient in FP64.  Tolerances (stated
once, used below):
  * IEEE-only operators (+ - * / min max abs neg sqrt and the protected
    variants; CUDA and numpy both round these correctly): the gradient equals
    the FP32 emulator of the same bytecode (tests/emulate.py) to 1e-10 of the
    constant's absolute contribution scale `gabs` (mean over datapoints of
    |adjoint reaching the constant|, from the emulator) beyond the FP32
    rounding of the returned value, non-finite entries in the same places,
    and the MSE to 1e-6 relative.
  * Against the FP64 oracle, errors are measured in units of gabs, the scale
    of the FP32 rounding in the per-datapoint sum.  Smooth populations
    (add sub mul sin cos tanh atan neg exp): median <= 1e-6, 95th
    percentile <= 1e-4, 99th <= 1e-2.  Populations with every operator,
    restricted to expressions whose FP32 forward MSE is within 1e-5 of the
    FP64 MSE: median <= 1e-6, 95th percentile <= 1e-3.  A constant whose FP64
    gradient is finite and below 1e30 is finite on the device, up to 1% of
    the constants for smooth populations and 3% with every operator (an FP32
    overflow or underflow inside its adjoint chain: a partial such as
    1 / (2 sqrt(u)) at an FP32 u that rounded to 0).
"""
import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from emulate import MAX_TANGENT_CONSTS, adjoint_bytecode, tangent_bytecode
from oracle import oracle
from symbolic_regression_gpu_b200 import _lib
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.evaluator import compile_population
from symbolic_regression_gpu_b200.population import Population

pytestmark = pytest.mark.gpu

IEEE_BINARY = (1, 2, 3, 4, 6, 7, 8)
IEEE_UNARY = (18, 23, 24, 25, 26, 27)
SMOOTH_UNARY = (10, 11, 15, 21, 25, 32)


def _dataset(rng, V, N, lo=-3.0, hi=3.0):
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(lo, hi, size=(V, N))
    X[V] = X[0] * X[1 % V] + np.sin(X[V - 1]) + 0.1 * rng.standard_normal(N)
    return X


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-30)


def _scaled_err(g, g_ref, gabs):
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.abs(g.astype(np.float64) - g_ref) / np.maximum(gabs, 1e-300)


def _const_expr(pop):
    co = pop.constant_offsets()
    return np.repeat(np.arange(pop.num_exprs), np.diff(co))


def _emulate32(pop, X, V, reverse_only=False):
    """(mse [E], grad [C], gabs [C]) of the FP32 bytecode emulator: forward
    mode for expressions with at most MAX_TANGENT_CONSTS constants, reverse
    mode above (reverse for all with reverse_only), as the device evaluates
    them."""
    code, offs, _ = compile_population(pop, V)
    co = pop.constant_offsets()
    mse = np.empty(pop.num_exprs)
    g = np.empty(int(co[-1]))
    ga = np.empty(int(co[-1]))
    with np.errstate(all="ignore"):
        for e in range(pop.num_exprs):
            s = slice(co[e], co[e + 1])
            nc = int(co[e + 1] - co[e])
            forward = nc <= MAX_TANGENT_CONSTS and not reverse_only
            run = tangent_bytecode if forward else adjoint_bytecode
            mse[e], g[s], ga[s] = run(code[offs[e]:offs[e + 1]], X, V, nc, dtype=np.float32,
                                      with_abs=True)
    return mse, g, ga


@pytest.mark.parametrize("reverse_only", [False, True])
def test_grad_ieee_ops_match_fp32_emulator(evaluator, reverse_only):
    rng = np.random.default_rng(31)
    V, N = 3, 5_000
    X = _dataset(rng, V, N)
    gen = synth.TreeGen(rng, V, p_const=0.4, binary=IEEE_BINARY, unary=IEEE_UNARY)
    exprs = [gen.depth_tree(6, full=False) for _ in range(200)]
    exprs += [gen.sized_tree(int(L)) for L in rng.integers(40, 120, size=20)]
    pop = Population.from_lists(exprs)
    evaluator.set_data(X)
    mode = _lib.SR_GRAD_CHECKPOINT | (_lib.SR_GRAD_REVERSE_ONLY if reverse_only else 0)
    mse, g = evaluator.eval_grad(pop, mode=mode)
    mse_e, g_e, gabs = _emulate32(pop, X, V, reverse_only)
    assert np.array_equal(np.isfinite(g), np.isfinite(g_e))
    fin = np.isfinite(g) & np.isfinite(gabs)
    assert fin.sum() > 300
    # Only the FP64 summation order (<= N * 2^-53 of the scale) and the FP32
    # rounding of the returned gradient (half an ulp) differ.
    excess = np.abs(g[fin] - g_e[fin]) - 2.0**-24 * np.abs(g_e[fin])
    err = np.maximum(excess, 0) / np.maximum(gabs[fin], 1e-300)
    assert err.max() <= 1e-10, err.max()
    mf = np.isfinite(mse_e)
    assert np.array_equal(np.isfinite(mse), mf)
    assert np.max(_rel(mse[mf], mse_e[mf])) <= 1e-6


def test_grad_smooth_population(evaluator):
    rng = np.random.default_rng(21)
    V, N = 3, 20_000
    X = _dataset(rng, V, N)
    gen = synth.TreeGen(rng, V, p_const=0.4, unary=SMOOTH_UNARY, binary=(1, 2, 3))
    pop = Population.from_lists([gen.depth_tree(6, full=False) for _ in range(300)])
    evaluator.set_data(X)
    mse, g = evaluator.eval_grad(pop)
    mse_o, g_o, gabs = oracle.grad_f64(pop, X, with_abs=True)
    fm = np.isfinite(mse_o)
    assert np.median(_rel(mse[fm], mse_o[fm])) <= 1e-6
    in_range = np.isfinite(g_o) & (np.abs(g_o) < 1e30)
    assert np.mean(~np.isfinite(g[in_range])) <= 0.01
    sel = in_range & np.isfinite(g)
    assert sel.sum() > 400
    err = _scaled_err(g[sel], g_o[sel], gabs[sel])
    assert np.median(err) <= 1e-6, np.median(err)
    assert np.quantile(err, 0.95) <= 1e-4, np.quantile(err, 0.95)
    assert np.quantile(err, 0.99) <= 1e-2, np.quantile(err, 0.99)


@pytest.mark.parametrize("seed", [0, 1])
def test_grad_mixed_population(evaluator, seed):
    rng = np.random.default_rng(50 + seed)
    V, N = 4, 6_000
    X = _dataset(rng, V, N)
    gen = synth.TreeGen(rng, V, p_const=0.35, binary=(1, 2, 3, 4, 5, 6, 7, 8, 9),
                        unary=tuple(range(10, 28)) + (32,))
    exprs = [gen.depth_tree(6, full=False) for _ in range(400)]
    # Long programs: spills and several tape-length classes.
    exprs += [gen.sized_tree(int(L)) for L in rng.integers(60, 200, size=60)]
    pop = Population.from_lists(exprs)
    evaluator.set_data(X)
    mse, g = evaluator.eval_grad(pop)
    mse_o, g_o, gabs = oracle.grad_f64(pop, X, with_abs=True)
    fm = np.isfinite(mse_o) & np.isfinite(mse)
    assert np.median(_rel(mse[fm], mse_o[fm])) <= 1e-6
    well = np.zeros(pop.num_exprs, bool)
    well[fm] = _rel(mse[fm], mse_o[fm]) <= 1e-5
    sel = well[_const_expr(pop)] & np.isfinite(g_o) & (np.abs(g_o) < 1e30)
    assert np.mean(~np.isfinite(g[sel])) <= 0.03
    sel &= np.isfinite(g)
    assert sel.sum() > 300
    err = _scaled_err(g[sel], g_o[sel], gabs[sel])
    assert np.median(err) <= 1e-6, np.median(err)
    assert np.quantile(err, 0.95) <= 1e-3, np.quantile(err, 0.95)


def test_grad_matches_forward_mse(evaluator):
    w = synth.grad_workload(seed=7, E=512, N=40_000)
    evaluator.set_data(w.X)
    mse_g, _ = evaluator.eval_grad(w.population)
    mse_f = evaluator.eval_mse(w.population)
    fin = np.isfinite(mse_f)
    assert np.array_equal(fin, np.isfinite(mse_g))
    assert np.max(_rel(mse_g[fin], mse_f[fin])) <= 1e-5


def test_grad_constant_expression_exact(evaluator):
    # mse(c) = mean((c - y)^2), d/dc = 2 (c - mean(y)); ragged N.
    rng = np.random.default_rng(5)
    X = _dataset(rng, 2, 1_001)
    pop = Population.from_lists([([0], [1.5]), ([1, 0, -1], [0, 0.25, 0]),
                                 ([3, -1, -1], [0, 1, 0])])
    evaluator.set_data(X)
    mse, g = evaluator.eval_grad(pop)
    y = X[2].astype(np.float64)
    c = np.float64(np.float32(1.5))
    q = np.float64(np.float32(0.25))
    assert g.size == 2
    assert g[0] == pytest.approx(2 * (c - y.mean()), rel=1e-5)
    assert g[1] == pytest.approx(2 * np.mean(q + X[0].astype(np.float64) - y), rel=1e-5)
    assert mse[0] == pytest.approx(np.mean((c - y) ** 2), rel=1e-5)


def test_grad_no_constants_and_empty(evaluator):
    rng = np.random.default_rng(6)
    X = _dataset(rng, 2, 500)
    evaluator.set_data(X)
    pop = Population.from_lists([([3, -1, -1], [0, 0, 1]), ([10, -1], [0, 1])])
    mse, g = evaluator.eval_grad(pop)
    assert g.size == 0
    mse_o, _ = oracle.mse_f64(pop, X)
    np.testing.assert_allclose(mse, mse_o, rtol=1e-5)
    mse, g = evaluator.eval_grad(Population.from_lists([]))
    assert mse.size == 0 and g.size == 0


def test_grad_too_many_constants_is_rejected(evaluator):
    rng = np.random.default_rng(8)
    evaluator.set_data(_dataset(rng, 2, 256))
    t, v = [0], [1.0]
    for k in range(70):
        t, v = [1] + t + [0], [0] + v + [float(k)]
    with pytest.raises(sg.SrError) as ei:
        evaluator.eval_grad(Population.from_lists([(t, v)]), mode=_lib.SR_GRAD_CHECKPOINT)
    assert ei.value.status == _lib.SR_ERR_UNSUPPORTED


def test_adam_lowers_mse_and_writes_constants_back(evaluator):
    w = synth.grad_workload(seed=9, E=256, N=50_000)
    pop = w.population
    evaluator.set_data(w.X)
    mse0 = evaluator.eval_mse(pop)
    consts, mse = evaluator.optimize_constants(pop, steps=20, lr=0.05)
    fin = np.isfinite(mse0) & np.isfinite(mse)
    # The returned MSE is the MSE at the returned constants.
    mse_chk = evaluator.eval_mse(pop.with_constants(consts.astype(np.float64)))
    np.testing.assert_allclose(mse[fin], mse_chk[fin], rtol=1e-5)
    # Expressions seeded with the perturbed hidden structure improve a lot.
    seeded = np.arange(0, pop.num_exprs, 4)
    assert np.median(mse[seeded] / mse0[seeded]) < 0.5
    assert np.mean(mse[fin] <= mse0[fin] * (1 + 1e-6)) > 0.8


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


@pytest.mark.parametrize("seed", [0, 1])
def test_recompute_matches_checkpoint(evaluator, seed):
    # Same values and partials, same sweep order: identical MSE, gradients
    # equal up to the order of the FP64 atomic adds across spans (<= 2 ulp of
    # the FP32 result).  Long programs give several segments, with spills.
    rng = np.random.default_rng(70 + seed)
    V, N = 4, 5_000
    X = _dataset(rng, V, N)
    gen = synth.TreeGen(rng, V, p_const=0.35, binary=(1, 2, 3, 4, 6, 7, 8),
                        unary=(10, 11, 15, 21, 25, 32, 22, 27))
    exprs = [gen.depth_tree(5, full=False) for _ in range(200)]
    exprs += [gen.sized_tree(int(L)) for L in rng.integers(40, 400, size=40)]
    pop = Population.from_lists(exprs)
    evaluator.set_data(X)
    m_c, g_c = evaluator.eval_grad(pop, mode=_lib.SR_GRAD_CHECKPOINT)
    m_r, g_r = evaluator.eval_grad(pop, mode=_lib.SR_GRAD_RECOMPUTE)
    assert np.array_equal(m_c, m_r, equal_nan=True)
    assert np.array_equal(np.isfinite(g_c), np.isfinite(g_r))
    fin = np.isfinite(g_c)
    assert _ulps(g_c[fin], g_r[fin]).max() <= 2


def test_recompute_adam(evaluator):
    w = synth.grad_workload(seed=11, E=128, N=20_000)
    evaluator.set_data(w.X)
    mse0 = evaluator.eval_mse(w.population)
    c_c, m_c = evaluator.optimize_constants(w.population, steps=5, mode=_lib.SR_GRAD_CHECKPOINT)
    c_r, m_r = evaluator.optimize_constants(w.population, steps=5, mode=_lib.SR_GRAD_RECOMPUTE)
    fin = np.isfinite(m_c) & np.isfinite(m_r)
    np.testing.assert_allclose(m_r[fin], m_c[fin], rtol=1e-4)
    seeded = np.arange(0, w.population.num_exprs, 4)
    assert np.median(m_r[seeded] / mse0[seeded]) < 1.0


def test_forward_and_reverse_modes_agree(evaluator):
    """The same population differentiated in forward mode (its expressions
    have at most 8 constants) and with SR_GRAD_REVERSE_ONLY: the same partials
    multiplied in opposite orders, so gradients agree to FP32 rounding of the
    per-datapoint products (1e-5 of the constant's contribution scale gabs)
    where both are finite, and finiteness differs for under 1% of the
    constants (an intermediate overflow in one order only)."""
    w = synth.grad_workload(seed=9, E=300, N=20_000)
    pop = w.population
    assert int(pop.constant_counts().max()) <= MAX_TANGENT_CONSTS
    evaluator.set_data(w.X)
    mse_f, g_f = evaluator.eval_grad(pop, mode=_lib.SR_GRAD_CHECKPOINT)
    mse_r, g_r = evaluator.eval_grad(pop, mode=_lib.SR_GRAD_CHECKPOINT | _lib.SR_GRAD_REVERSE_ONLY)
    fm = np.isfinite(mse_f)
    assert np.array_equal(fm, np.isfinite(mse_r))
    assert np.max(_rel(mse_f[fm], mse_r[fm])) <= 1e-6
    _, _, gabs = _emulate32(pop, w.X, w.num_vars, reverse_only=True)
    both = np.isfinite(g_f) & np.isfinite(g_r) & np.isfinite(gabs)
    assert np.mean(np.isfinite(g_f) != np.isfinite(g_r)) <= 0.01
    assert both.sum() > 500
    err = _scaled_err(g_f[both], g_r[both].astype(np.float64), gabs[both])
    assert err.max() <= 1e-5, err.max()


def test_forward_mode_long_programs_match_fp32_emulator(evaluator):
    """Forward mode on long programs (60-127 tokens, deep Sethi-Ullman spills,
    spill slots beyond the ones kept in shared memory) with at most 8
    constants, IEEE operators only: the same exactness as the short programs
    against the FP32 emulator."""
    rng = np.random.default_rng(44)
    V, N = 3, 4_000
    X = _dataset(rng, V, N)
    gen = synth.TreeGen(rng, V, p_const=0.05, binary=IEEE_BINARY, unary=IEEE_UNARY)
    full = synth.TreeGen(rng, V, p_const=0.05, binary=IEEE_BINARY, unary=IEEE_UNARY,
                         p_unary=0.0)
    exprs = []
    while len(exprs) < 120:
        # full binary trees of depth 6 (127 tokens, 6 spill slots) and random shapes
        e = full.depth_tree(6, full=True) if len(exprs) % 2 else gen.sized_tree(
            int(rng.integers(60, 128)))
        if 1 <= sum(1 for tk in e[0] if tk == 0) <= MAX_TANGENT_CONSTS:
            exprs.append(e)
    pop = Population.from_lists(exprs)
    _, _, slots = compile_population(pop, V)
    assert int(slots.max()) >= 5  # beyond the spill slots kept in shared memory
    evaluator.set_data(X)
    mse, g = evaluator.eval_grad(pop)
    mse_e, g_e, gabs = _emulate32(pop, X, V)
    assert np.array_equal(np.isfinite(g), np.isfinite(g_e))
    fin = np.isfinite(g) & np.isfinite(gabs)
    assert fin.sum() > 200
    excess = np.abs(g[fin] - g_e[fin]) - 2.0**-24 * np.abs(g_e[fin])
    err = np.maximum(excess, 0) / np.maximum(gabs[fin], 1e-300)
    assert err.max() <= 1e-10, err.max()
    mf = np.isfinite(mse_e)
    assert np.array_equal(np.isfinite(mse), mf)
    assert np.max(_rel(mse[mf], mse_e[mf])) <= 1e-6
