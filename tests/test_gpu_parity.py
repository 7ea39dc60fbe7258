"""CUDA path against the reference's outputs (golden vectors) and the oracle.

Tolerances (stated once, used below):
  * IEEE operations (+ - * / sqrt, reciprocal, min/max, abs, neg, protected
    variants): bit-identical predictions.
  * Single transcendental operators: <= 4 ulp of glibc's result per datapoint.
  * Compound expressions: the condition-aware rule (oracle.datapoint_parity /
    oracle.mse_parity, defined and tested on the CPU in tests/test_parity_rule.py).
    Every datapoint lies within max(4 ulp, B) of the reference's value and
    agrees on being finite, where B is the running forward error bound of the
    expression at that datapoint built from the documented maximum errors of
    CUDA's and glibc's functions (B = 0 for IEEE-only expressions); every
    MSE lies within max(1e-6, its bound) relative of the reference's.  Only
    datapoints whose bound reaches a discontinuity, singularity or overflow
    (flagged), and the expressions holding one, are exempt; the exempt shares
    are printed.
  * Reduction error (GPU MSE vs FP64 sum of the GPU's own FP32 predictions):
    <= oracle.REDUCTION_REL (2.5e-7) relative, the worst case of the device's
    summation order.
  * Against the FP64 evaluation: every MSE within max(1e-5, its bound)
    (mode 1 of the same rule: the FP32 evaluation's own rounding).
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle
import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import opcodes as op
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.population import Population

pytestmark = pytest.mark.gpu

IEEE_OPS = {op.ADD, op.SUB, op.MUL, op.DIV, op.MIN, op.MAX, op.LOOSE_DIV, op.INV,
            op.LOOSE_INV, op.ABS, op.NEG, op.SQRT, op.LOOSE_SQRT}


def ordered(x):
    i = np.asarray(x, np.float32).view(np.int32).astype(np.int64)
    return np.where(i < 0, -(i & 0x7FFFFFFF), i)


def ulp(a, b):
    return np.abs(ordered(a) - ordered(b))


def same_float(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-30)


def ieee_only(pop):
    return np.array([set(t[t > 0].tolist()) <= IEEE_OPS for t, _ in pop])


def test_single_operator_predictions(evaluator):
    pop, d = load_golden("eval_all_ops.npz")
    n_edge = 31
    edge = pop.slice(0, n_edge)
    evaluator.set_data(d["X"])
    pred = evaluator.predictions(edge)
    ref = d["pred"][:n_edge]
    for i, (t, _) in enumerate(edge):
        ops = set(t[t > 0].tolist())
        nan_g, nan_r = np.isnan(pred[i]), np.isnan(ref[i])
        assert (nan_g == nan_r).all(), f"expr {i} {t}: NaN pattern differs"
        fin = np.isfinite(ref[i]) & np.isfinite(pred[i])
        assert (np.isinf(pred[i]) == np.isinf(ref[i])).all(), f"expr {i}: Inf pattern differs"
        if ops <= IEEE_OPS:
            assert same_float(pred[i], ref[i]).all(), f"expr {i} {t}: not bit-identical"
        else:
            worst = int(ulp(pred[i][fin], ref[i][fin]).max(initial=0))
            assert worst <= 4, f"expr {i} {t}: {worst} ulp"


def _assert_datapoint_rule(pop, X, pred, ref, label):
    b = oracle.error_bound(pop, X, mode=0, per_datapoint=True)
    fin = np.isfinite(ref)
    # the bound's centre is the reference's own value
    assert (b["pred"][fin].astype(np.float32) == ref[fin]).all()
    r = oracle.datapoint_parity(pred, ref, b["bound"], b["flag"])
    n = r["datapoints"]
    print(f"{label}: {r['bit_identical'] / n:.4f} bit-identical, {r['within_bar'] / n:.4f} "
          f"within 4 ulp, exempt: {r['exempt_flagged'] / n:.4f} flagged, "
          f"{r['exempt_conditioning'] / n:.4f} by conditioning (bound > 4 ulp)")
    assert r["violations"] == 0, r
    return r


def _assert_mse_rule(pop, X, mse, ref_mse, label, mode=0, bar=oracle.MSE_BAR):
    b = oracle.error_bound(pop, X, mode=mode)
    r = oracle.mse_parity(mse, ref_mse, b["mse_bound"], b["flagged"], bar=bar)
    n = max(r["expressions"], 1)
    print(f"{label}: within {bar:g}: {r['within_bar_all']:.4f} of all, "
          f"{r['within_bar_well_conditioned']:.4f} of the well-conditioned; exempt: "
          f"{r['exempt_flagged'] / n:.4f} flagged, {r['exempt_conditioning'] / n:.4f} by "
          f"conditioning")
    assert r["violations"] == 0, r
    assert r["within_bar_well_conditioned"] == 1.0
    return r, b


def test_random_all_ops_predictions(evaluator):
    pop, d = load_golden("eval_all_ops.npz")
    evaluator.set_data(d["X"])
    pred = evaluator.predictions(pop)
    _assert_datapoint_rule(pop, d["X"], pred, d["pred"], "all-ops random trees")
    ieee = ieee_only(pop)
    assert same_float(pred[ieee], d["pred"][ieee]).all()


def test_workload_ops_predictions_vs_oracle(evaluator):
    w = synth.plain_workload(seed=11, E=200, N=4096)
    evaluator.set_data(w.X)
    pred = evaluator.predictions(w.population)
    ref = oracle.predict_f32(w.population, w.X)
    r = _assert_datapoint_rule(w.population, w.X, pred, ref, "workload trees vs oracle")
    assert r["bit_identical"] / r["datapoints"] >= 0.5


def test_mse_vs_reference_golden(evaluator):
    pop, d = load_golden("eval_workload_ops.npz")
    evaluator.set_data(d["X"])
    mse = evaluator.eval_mse(pop)
    ref = d["mse"]
    assert (np.isnan(mse) == np.isnan(ref)).all()
    _assert_mse_rule(pop, d["X"], mse, ref, "MSE vs reference CPU")
    ieee = ieee_only(pop) & np.isfinite(ref)
    assert (rel(mse[ieee], ref[ieee]) <= 1e-6).all()


def test_exp_clamp_goldens(evaluator):
    """Opcode 32 (exp clamped at 80) against the reference evaluator with the
    one added case, at arguments around 80, 88.7 and 100 and in random
    workload expressions."""
    pop, d = load_golden("eval_exp_clamp.npz")
    evaluator.set_data(d["X"])
    pred = evaluator.predictions(pop)
    _assert_datapoint_rule(pop, d["X"], pred, d["pred"], "exp clamp edge expressions")
    mse = evaluator.eval_mse(pop)
    _assert_mse_rule(pop, d["X"], mse, d["mse"], "exp clamp edge MSE")
    w = Population(d["w_tokens"], d["w_values"], d["w_offsets"])
    evaluator.set_data(d["w_X"])
    wm = evaluator.eval_mse(w)
    assert (np.isnan(wm) == np.isnan(d["w_mse"])).all()
    _assert_mse_rule(w, d["w_X"], wm, d["w_mse"], "exp clamp workload MSE")
    E, N = int(d["w_pred_E"]), int(d["w_pred_N"])
    sub, Xs = w.slice(0, E), d["w_X"][:, :N].copy()
    evaluator.set_data(Xs)
    _assert_datapoint_rule(sub, Xs, evaluator.predictions(sub), d["w_pred"],
                           "exp clamp workload trees")


def test_plain_workload_full_size(evaluator):
    """The plain-forward workload at its full size (1,000 expressions x 100,000
    datapoints) against the reference's MSEs (the reference evaluator with the
    exp-clamp case where it is built here, else its restatement, which the
    goldens pin bit for bit), under the rule; per datapoint on the first
    4,096 datapoints of every expression."""
    w = synth.plain_workload(seed=1, E=1000, N=100_000)
    evaluator.set_data(w.X)
    mse = evaluator.eval_mse(w.population)
    ref = oracle.mse_f32(w.population, w.X)
    if oracle.reference_expc_available():
        refx, _ = oracle.refx_mse(w.population, w.X)
        assert same_float(refx, ref).all()
    assert (np.isnan(mse) == np.isnan(ref)).all()
    r, b = _assert_mse_rule(w.population, w.X, mse, ref, "plain workload 1000 x 100k")
    assert same_float(b["mse"].astype(np.float32), ref).all()
    Xs = w.X[:, :4096].copy()
    evaluator.set_data(Xs)
    _assert_datapoint_rule(w.population, Xs, evaluator.predictions(w.population),
                           oracle.predict_f32(w.population, Xs), "plain workload per datapoint")


def test_mse_all_ops_vs_reference_golden(evaluator):
    pop, d = load_golden("eval_all_ops.npz")
    evaluator.set_data(d["X"])
    mse = evaluator.eval_mse(pop)
    ref = d["mse"]
    assert (np.isnan(mse) == np.isnan(ref)).all()
    assert (np.isinf(mse) == np.isinf(ref)).all()
    ieee = ieee_only(pop) & np.isfinite(ref)
    assert (rel(mse[ieee], ref[ieee]) <= 1e-6).all()


def test_reduction_error(evaluator):
    w = synth.plain_workload(seed=12, E=120, N=50_000)
    evaluator.set_data(w.X)
    pred = evaluator.predictions(w.population)
    mse = evaluator.eval_mse(w.population)
    want = oracle.mse_of_predictions(pred, w.X[-1])
    assert (np.isnan(mse) == np.isnan(want)).all()
    ok = np.isfinite(want)
    assert (rel(mse[ok], want[ok]) <= oracle.REDUCTION_REL).all(), rel(mse[ok], want[ok]).max()


def test_mse_vs_fp64_oracle(evaluator):
    w = synth.plain_workload(seed=13, E=200, N=20_000)
    evaluator.set_data(w.X)
    mse = evaluator.eval_mse(w.population)
    m64, cnt = oracle.mse_f64(w.population, w.X)
    _assert_mse_rule(w.population, w.X, mse, m64, "FP32 vs FP64", mode=1, bar=oracle.FP64_BAR)


@pytest.mark.parametrize("dpt,warps", [(4, 1), (4, 8), (8, 3), (8, 8), (8, 15), (8, 31)])
def test_launch_shapes_agree(dpt, warps):
    w = synth.plain_workload(seed=14, E=77, N=3001)
    ref = oracle.mse_f32(w.population, w.X)
    with sg.Evaluator(device=0, dpt=dpt, warps_per_block=warps) as ev:
        ev.set_data(w.X)
        mse = ev.eval_mse(w.population)
        pred = ev.predictions(w.population)
    base = oracle.predict_f32(w.population, w.X)
    ieee = ieee_only(w.population)
    assert same_float(pred[ieee], base[ieee]).all()
    ok = np.isfinite(ref)
    assert (np.isnan(mse) == np.isnan(ref)).all()
    assert np.median(rel(mse[ok], ref[ok])) <= 1e-7


def test_plain_kernel_matches_batched(evaluator):
    w = synth.plain_workload(seed=15, E=150, N=10_000)
    evaluator.set_data(w.X)
    a = evaluator.eval_mse(w.population)
    b = evaluator.eval_mse(w.population, plain=True)
    assert (np.isnan(a) == np.isnan(b)).all()
    ok = np.isfinite(a)
    assert (rel(a[ok], b[ok]) <= 1e-6).all()


@pytest.mark.parametrize("N", [1, 2, 127, 255, 256, 257, 1023, 1025, 4097, 70_001])
def test_ragged_sizes(evaluator, N):
    # Masking / indexing at every datapoint count: the MSE must be the FP64
    # reduction of the GPU's own predictions, and the predictions must agree
    # with the oracle (IEEE-only expressions bit for bit).
    w = synth.plain_workload(seed=16, E=37, N=N)
    evaluator.set_data(w.X)
    mse = evaluator.eval_mse(w.population)
    pred = evaluator.predictions(w.population)
    assert pred.shape == (37, N)
    want = oracle.mse_of_predictions(pred, w.X[-1])
    assert (np.isnan(mse) == np.isnan(want)).all()
    ok = np.isfinite(want)
    assert (rel(mse[ok], want[ok]) <= oracle.REDUCTION_REL).all()
    ref = oracle.predict_f32(w.population, w.X)
    ieee = ieee_only(w.population)
    assert same_float(pred[ieee], ref[ieee]).all()
    assert (np.isnan(pred) == np.isnan(ref)).mean() >= 0.999


@pytest.mark.parametrize("V", [10, 20, 31])
def test_wide_datasets_shrink_span(V):
    # Many variables force a smaller span; every datapoint must still count.
    rng = np.random.default_rng(V)
    N = 5000
    X = rng.uniform(-2, 2, size=(V + 1, N)).astype(np.float32)
    gen = synth.TreeGen(rng, V, binary=(op.ADD, op.SUB, op.MUL), unary=(op.NEG, op.ABS))
    pop = Population.from_lists([gen.sized_tree(int(L)) for L in rng.integers(1, 400, 30)])
    for dpt, warps in [(4, 8), (8, 8), (8, 16), (8, 31)]:
        with sg.Evaluator(device=0, dpt=dpt, warps_per_block=warps) as ev:
            ev.set_data(X)
            pred = ev.predictions(pop)
            mse = ev.eval_mse(pop)
        assert same_float(pred, oracle.predict_f32(pop, X)).all(), (V, dpt, warps)
        want = oracle.mse_of_predictions(pred, X[-1])
        ok = np.isfinite(want)
        assert (rel(mse[ok], want[ok]) <= oracle.REDUCTION_REL).all(), (V, dpt, warps)


@pytest.mark.parametrize("V,want_warps", [(5, 31), (31, 8)])
def test_default_launch_shape(V, want_warps):
    # The untuned shape for the protected profile is one 1,024-thread block
    # per SM (31 evaluating warps) unless its shared memory does not fit even
    # at 512-datapoint spans (many variables), then 8 warps at 3 blocks per SM.
    rng = np.random.default_rng(100 + V)
    N = 20_000
    X = rng.uniform(-2, 2, size=(V + 1, N)).astype(np.float32)
    gen = synth.TreeGen(rng, V, binary=(op.ADD, op.SUB, op.MUL), unary=(op.SIN, op.COS))
    exprs = [gen.sized_tree(int(L)) for L in rng.integers(3, 64, 300)]
    exprs += [gen.depth_tree(5, full=True) for _ in range(4)]  # 3 spill slots
    pop = Population.from_lists(exprs)
    # With 3 spill slots per warp in shared memory, 31 warps and 32 data rows
    # need more than 227 KB at 512-datapoint spans.
    assert sg.evaluator.compile_population(pop, V)[2].max() >= 3
    with sg.Evaluator(device=0) as ev:
        ev.set_data(X)
        mse = ev.eval_mse(pop)
        assert (ev.stats.dpt, ev.stats.warps_per_block) == (8, want_warps)
        pred = ev.predictions(pop)
    want = oracle.mse_of_predictions(pred, X[-1])
    ok = np.isfinite(want)
    assert (np.isnan(mse) == np.isnan(want)).all()
    assert (rel(mse[ok], want[ok]) <= oracle.REDUCTION_REL).all()


def test_zero_datapoints_gives_nan(evaluator):
    X = np.zeros((3, 0), np.float32)
    evaluator.set_data(X)
    pop = Population.from_lists([([op.ADD, -1, 0], [0, 0, 1.0])])
    assert np.isnan(evaluator.eval_mse(pop)).all()


def test_empty_population(evaluator):
    w = synth.plain_workload(seed=17, E=3, N=100)
    evaluator.set_data(w.X)
    empty = Population(np.zeros(0, np.int32), np.zeros(0), np.zeros(1, np.int64))
    assert evaluator.eval_mse(empty).shape == (0,)


def test_longest_expression_and_extreme_var_counts(evaluator):
    import sys
    sys.setrecursionlimit(max(sys.getrecursionlimit(), 10_000))
    rng = np.random.default_rng(18)
    for V in (0, 1, 31):
        N = 700
        X = rng.uniform(-2, 2, size=(V + 1, N)).astype(np.float32)
        gen = synth.TreeGen(rng, V)
        ieee = synth.TreeGen(rng, V, binary=(op.ADD, op.SUB, op.MUL, op.LOOSE_DIV),
                             unary=(op.LOOSE_SQRT, op.NEG, op.ABS))
        exprs = [ieee.sized_tree(1000), gen.sized_tree(1), gen.sized_tree(3)]
        # a deep left-leaning chain: raw stack depth 1 but 1023 tokens
        t = [op.ADD] * 511 + [op.TOK_CONST] * 512
        exprs.append((t, [0.0] * 511 + list(rng.uniform(-1, 1, 512))))
        pop = Population.from_lists(exprs)
        evaluator.set_data(X)
        mse = evaluator.eval_mse(pop)
        ref = oracle.mse_f32(pop, X)
        assert (np.isnan(mse) == np.isnan(ref)).all()
        ok = np.isfinite(ref)
        assert (rel(mse[ok], ref[ok]) <= 1e-4).all(), (V, mse, ref)


def test_invalid_datapoints_masked(evaluator):
    X = np.array([[0.0, 1.0, -1.0, 2.0], [0.0, 0.0, 0.0, 0.0]], np.float32)
    evaluator.set_data(X)
    pop = Population.from_lists([
        ([op.DIV, op.TOK_CONST, op.TOK_VAR], [0, 1.0, 0]),    # 1/x: NaN? no: Inf at x=0
        ([op.LOG, op.TOK_VAR], [0, 0]),                       # NaN for x<0, -Inf at 0
        ([op.DIV, op.TOK_VAR, op.TOK_CONST], [0, 0, 0.0]),    # always NaN
        ([op.MUL, op.TOK_CONST, op.TOK_VAR], [0, 3e19, 0]),   # square overflows -> Inf
    ])
    mse = evaluator.eval_mse(pop)
    ref = oracle.mse_f32(pop, X)
    assert same_float(mse, ref).all(), (mse, ref)
    assert np.isnan(mse[2]) and np.isinf(mse[3])


def test_prepare_launch_read_is_repeatable(evaluator):
    w = synth.plain_workload(seed=19, E=64, N=20_000)
    evaluator.set_data(w.X)
    evaluator.prepare(w.population)
    outs = []
    for _ in range(3):
        evaluator.launch()
        outs.append(evaluator.read_mse())
    assert same_float(outs[0], outs[1]).all() and same_float(outs[1], outs[2]).all()
    assert evaluator.stats.kernel_launches >= 2
    assert evaluator.stats.node_evals == w.population.num_tokens * w.num_dps


def test_bad_input_reports_status(evaluator):
    w = synth.plain_workload(seed=20, E=4, N=100)
    evaluator.set_data(w.X)
    bad = Population.from_lists([([op.ADD, -1], [0, 0])])
    with pytest.raises(sg.SrError) as ei:
        evaluator.eval_mse(bad)
    assert ei.value.status == sg._lib.SR_ERR_MALFORMED_EXPRESSION
    # the context stays usable
    assert np.isfinite(evaluator.eval_mse(w.population)).any()


def test_ieee_only_long_trees_bit_exact(evaluator):
    """Structural check of the device interpreter: with IEEE operators only,
    every prediction is bit-identical to right-to-left prefix evaluation,
    for long trees and trees that need many spill slots."""
    import sys
    sys.setrecursionlimit(max(sys.getrecursionlimit(), 10_000))
    rng = np.random.default_rng(21)
    V = 3
    X = rng.uniform(-2, 2, size=(V + 1, 3000)).astype(np.float32)
    gen = synth.TreeGen(rng, V, binary=(op.ADD, op.SUB, op.MUL, op.LOOSE_DIV, op.MIN, op.MAX),
                        unary=(op.LOOSE_SQRT, op.NEG, op.ABS, op.LOOSE_INV))
    exprs = [gen.sized_tree(int(L)) for L in rng.integers(1, 1025, 60)]

    def full(depth):
        if depth == 0:
            return [op.LOOSE_SQRT, -1], [0.0, float(rng.integers(V))]
        a, b = full(depth - 1), full(depth - 1)
        return [op.SUB] + a[0] + b[0], [0.0] + a[1] + b[1]
    for d in range(1, 9):
        exprs.append(full(d))
    pop = Population.from_lists(exprs)
    evaluator.set_data(X)
    pred = evaluator.predictions(pop)
    ref = oracle.predict_f32(pop, X)
    bad = [i for i in range(pop.num_exprs) if not same_float(pred[i], ref[i]).all()]
    assert not bad, bad


def test_operator_profiles_give_identical_results():
    """A launch dominated by the protected operator set runs the kOpsProtected
    interpreter (other operators out of line), a mixed one kOpsAll: the same
    expression gets the same MSE bits either way."""
    rng = np.random.default_rng(77)
    V, N = 3, 20_000
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(-3, 3, size=(V, N))
    X[V] = np.sin(X[0]) * X[1] + 0.1
    prot = synth.TreeGen(rng, V, p_const=0.3, binary=(1, 2, 3, 8), unary=(10, 11, 32, 22, 27))
    rare = synth.TreeGen(rng, V, p_const=0.3, binary=(4, 5, 6, 7, 9), unary=tuple(range(12, 22)))
    mixed = synth.TreeGen(rng, V, p_const=0.3, binary=tuple(range(1, 10)),
                          unary=tuple(range(10, 28)) + (32,))
    base = [prot.depth_tree(6, full=False) for _ in range(400)]
    base += [mixed.depth_tree(4, full=False) for _ in range(8)]   # a few rare operators
    extra = [rare.depth_tree(6, full=False) for _ in range(600)]
    # one launch shape for both (the untuned default shape depends on the
    # profile, and the shape sets the summation order)
    with sg.Evaluator(device=0, dpt=8, warps_per_block=8) as ev:
        ev.set_data(X)
        a = ev.eval_mse(Population.from_lists(base))
        b = ev.eval_mse(Population.from_lists(base + extra))[:len(base)]
    same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    assert same.all()


@pytest.mark.parametrize("split", [0, 2, 7])
def test_spill_split_gives_identical_results(split):
    """Spill slots kept in shared memory or in global scratch (the split the
    autotuner chooses) hold the same values: identical MSE bits."""
    rng = np.random.default_rng(5)
    V, N = 3, 20_000
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(-2, 2, size=(V, N))
    X[V] = X[0] * X[1] - X[2]
    gen = synth.TreeGen(rng, V, binary=(1, 2, 3, 8), unary=(10, 11), p_const=0.3, p_unary=0.0)
    pop = Population.from_lists([gen.depth_tree(8, full=True) for _ in range(48)]
                                + [gen.depth_tree(5, full=False) for _ in range(200)])
    with sg.Evaluator(device=0, dpt=8, warps_per_block=8) as ev:
        ev.set_data(X)
        want = ev.eval_mse(pop)
    with sg.Evaluator(device=0, dpt=8, warps_per_block=8, smem_spill_slots=split) as ev:
        ev.set_data(X)
        got = ev.eval_mse(pop)
    assert ((got.view(np.uint32) == want.view(np.uint32)) | (np.isnan(got) & np.isnan(want))).all()


def test_autotuner_records_the_spill_split(tmp_path):
    rng = np.random.default_rng(6)
    V, N = 3, 50_000
    X = rng.uniform(-2, 2, size=(V + 1, N)).astype(np.float32)
    gen = synth.TreeGen(rng, V, binary=(1, 2, 3, 8), unary=(10, 11), p_const=0.3, p_unary=0.0)
    pop = Population.from_lists([gen.depth_tree(7, full=True) for _ in range(300)])
    path = tmp_path / "tune.json"
    with sg.Evaluator(device=0, autotune=True, tune_cache_path=str(path)) as ev:
        ev.set_data(X)
        a = ev.eval_mse(pop)
    entries = [ln for ln in path.read_text().splitlines() if ln.strip().startswith('"')]
    assert len(entries) == 1
    shape = [int(x) for x in entries[0].split("[")[1].split("]")[0].split(",")]
    assert len(shape) == 4 and shape[0] in (4, 8, 16) and -1 <= shape[2] <= 16
    assert shape[3] in (2, 4, 8)
    # a new context reads the tuned shape back and gives the same result
    with sg.Evaluator(device=0, autotune=True, tune_cache_path=str(path)) as ev:
        ev.set_data(X)
        b = ev.eval_mse(pop)
    assert ((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all()
