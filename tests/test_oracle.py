"""The C restatement (oracle/sr_oracle.c) against the reference's own outputs
(tests/golden, produced by tests/golden/make_golden.py)."""
import numpy as np

from conftest import load_golden
from oracle import oracle
from symbolic_regression_gpu_b200 import opcodes as op


def _same_float(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))


def test_predictions_all_ops_bit_exact():
    pop, d = load_golden("eval_all_ops.npz")
    pred = oracle.predict_f32(pop, d["X"], threads=2)
    assert pred.shape == d["pred"].shape
    assert _same_float(pred, d["pred"]).all()


def test_mse_all_ops_bit_exact():
    pop, d = load_golden("eval_all_ops.npz")
    mse = oracle.mse_f32(pop, d["X"], threads=3)
    assert _same_float(mse, d["mse"]).all()


def test_workload_ops_mse_and_predictions():
    pop, d = load_golden("eval_workload_ops.npz")
    mse = oracle.mse_f32(pop, d["X"], threads=4)
    assert _same_float(mse, d["mse"]).all()
    E, N = int(d["pred_E"]), int(d["pred_N"])
    pred = oracle.predict_f32(pop.slice(0, E), d["X"][:, :N].copy(), threads=2)
    assert _same_float(pred, d["pred"]).all()


def test_exp_clamp_extension_semantics():
    # expf(fminf(x, 80)): identical to the reference EXP below 80, constant above.
    for x in [-100.0, -1.0, 0.0, 1.5, 79.99, 80.0, 80.5, 1e30, float("inf")]:
        want = oracle.op_f32(op.EXP, min(x, 80.0))
        assert oracle.op_f32(op.EXP_CLAMP, x) == want
    assert np.isfinite(oracle.op_f32(op.EXP_CLAMP, 1e30))
    # NaN: fminf(NaN, 80) = 80.
    assert oracle.op_f32(op.EXP_CLAMP, float("nan")) == oracle.op_f32(op.EXP, 80.0)


def test_fp64_oracle_agrees_with_float_path_on_benign_inputs():
    pop, d = load_golden("eval_workload_ops.npz")
    mse32 = d["mse"].astype(np.float64)
    mse64, cnt = oracle.mse_f64(pop, d["X"], threads=4)
    ok = np.isfinite(mse32) & np.isfinite(mse64) & (cnt == d["X"].shape[1])
    rel = np.abs(mse64[ok] - mse32[ok]) / np.maximum(np.abs(mse64[ok]), 1e-30)
    # FP32 evaluation error of random expressions: small for most of them.
    assert np.median(rel) < 1e-5


def test_keys_and_merkle_match_reference():
    pop, d = load_golden("hash_kat.npz")
    sizes, merkle, keys = [], [], []
    for t, v in pop:
        s, h = oracle.merkle(t, v)
        sizes.append(s)
        merkle.append(h)
        for i in range(t.size):
            keys.append(oracle.flat_key(t[i:i + s[i]], v[i:i + s[i]]))
    assert (np.concatenate(sizes) == d["sizes"]).all()
    assert (np.concatenate(merkle) == d["merkle"]).all()
    assert (np.array(keys, np.uint64) == d["flat_keys"]).all()
    # The reference's two flat-key functions agree with each other.
    assert (d["flat_keys"] == d["flat_keys_gpu_path"]).all()


def test_planted_mistake_is_caught():
    """A deliberately wrong oracle (on the CPU) must fail the comparison."""
    pop, d = load_golden("eval_all_ops.npz")
    pred = oracle.predict_f32(pop, d["X"], threads=2)
    pred[5, 7] = np.nextafter(pred[5, 7], np.float32(np.inf)) if np.isfinite(pred[5, 7]) else 1.0
    assert not _same_float(pred, d["pred"]).all()


def _load_exp_clamp():
    from symbolic_regression_gpu_b200.population import Population
    pop, d = load_golden("eval_exp_clamp.npz")
    w = Population(d["w_tokens"], d["w_values"], d["w_offsets"])
    return pop, w, d


def test_exp_clamp_goldens_bit_exact():
    """Opcode 32 at arguments around 80, 88.7 and 100, and the workload
    operators with opcode 32, against the reference evaluator with the one
    added case (tests/golden/make_golden.py)."""
    pop, w, d = _load_exp_clamp()
    assert _same_float(oracle.predict_f32(pop, d["X"], threads=2), d["pred"]).all()
    assert _same_float(oracle.mse_f32(pop, d["X"], threads=2), d["mse"]).all()
    assert _same_float(oracle.mse_f32(w, d["w_X"], threads=3), d["w_mse"]).all()
    E, N = int(d["w_pred_E"]), int(d["w_pred_N"])
    pred = oracle.predict_f32(w.slice(0, E), d["w_X"][:, :N].copy(), threads=2)
    assert _same_float(pred, d["w_pred"]).all()
    # The clamp: every argument at or above 80 gives expf(80).
    e80 = np.float32(oracle.op_f32(op.EXP, 80.0))
    x0 = d["X"][0]
    big = ~np.isnan(x0) & (x0 >= 80)
    assert (d["pred"][0][big] == e80).all() and big.sum() >= 10
    assert (d["pred"][0][np.isnan(x0)] == e80).all()
