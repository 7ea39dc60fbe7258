"""Generate the golden vectors under tests/golden/ from the reference itself.

Runs the reference's CPU evaluator (evaluate_single_expr / evaluate_cpu_mse,
src/cleaned/cl_cpu_eval.cpp), its subtree hashing and detection
(src/utils/detect.cpp) and its cache marking (src/cleaned/cl_gpu_eval.cu:294-329),
all compiled unchanged into oracle/_ref/libref_oracle.so, and the same CPU
evaluator with the one added case for opcode 32 (exp clamped at 80,
oracle/_ref/libref_expc.so, see oracle/ref_expc_shim.cpp), on seeded inputs,
and stores inputs and outputs as .npz files.  The fixtures are committed; the
tests never need the reference tree.

    make -C oracle REF=<reference tree> ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from symbolic_regression_gpu_b200 import opcodes as op  # noqa: E402
from symbolic_regression_gpu_b200 import synth  # noqa: E402
from symbolic_regression_gpu_b200.population import Population  # noqa: E402

ALL_BINARY = list(op.BINARY_OPS)
ALL_UNARY = list(op.REFERENCE_UNARY_OPS)


def _edge_dataset(rng, V: int, N: int) -> np.ndarray:
    """Datapoints mixing ordinary values with zeros, signed zeros, tiny,
    huge and negative values, so protected operators take every branch."""
    X = rng.uniform(-4.0, 4.0, size=(V + 1, N)).astype(np.float32)
    special = np.array([0.0, -0.0, 1e-10, -1e-10, 1e-30, 3.0e38, -3.0e38, 1.0, -1.0,
                        80.0, 81.0, 100.0, -100.0, 1e-45, 0.5, np.pi], np.float32)
    for v in range(V):
        k = min(N, special.size)
        X[v, v:v + k] = np.roll(special, v)[:k]
    return X


def _edge_expressions(V: int):
    """Hand-written expressions that hit reference corner cases."""
    C, X = op.TOK_CONST, op.TOK_VAR
    return [
        ([X], [0.0]),                                  # single variable
        ([C], [2.5]),                                  # single constant
        ([X], [float(V)]),                             # index == V: CPU pushes 0
        ([X], [float(V + 7)]),                         # index > V
        ([op.DIV, X, C], [0.0, 0.0, 0.0]),             # x / 0 -> NaN
        ([op.LOOSE_DIV, X, C], [0.0, 1.0, 0.0]),       # protected division by 0
        ([op.LOOSE_DIV, C, X], [0.0, 1.0, 0.0]),
        ([op.LOOSE_INV, X], [0.0, 0.0]),
        ([op.LOOSE_LOG, X], [0.0, 0.0]),
        ([op.LOG, X], [0.0, 1.0]),
        ([op.SQRT, X], [0.0, 0.0]),
        ([op.LOOSE_SQRT, X], [0.0, 2.0]),
        ([op.POW, X, X], [0.0, 0.0, 1.0]),
        ([op.LOOSE_POW, X, C], [0.0, 0.0, 0.0]),       # 0^0 -> 0
        ([op.LOOSE_POW, C, C], [0.0, 0.0, 0.0]),
        ([op.EXP, X], [0.0, 0.0]),
        ([op.SUB, X, X], [0.0, 1.0, 0.0]),             # operand order
        ([op.DIV, X, X], [0.0, 1.0, 0.0]),
        ([op.MIN, op.DIV, X, C, X], [0.0, 0.0, 0.0, 0.0, 1.0]),  # NaN into fmin
        ([op.MAX, X, op.DIV, X, C], [0.0, 1.0, 0.0, 0.0, 0.0]),
        ([op.ASIN, X], [0.0, 0.0]),
        ([op.ACOS, X], [0.0, 1.0]),
        ([op.ATAN, X], [0.0, 0.0]),
        ([op.TAN, X], [0.0, 0.0]),
        ([op.SINH, X], [0.0, 1.0]),
        ([op.COSH, X], [0.0, 0.0]),
        ([op.TANH, X], [0.0, 1.0]),
        ([op.INV, X], [0.0, 0.0]),
        ([op.NEG, op.ABS, X], [0.0, 0.0, 1.0]),
        ([op.MUL, C, X], [0.0, 1.7, 0.0]),
        ([op.ADD, X, C], [0.0, 2.9, 1.0]),              # var index 2.9 -> 2
    ]


def _population_all_ops(seed: int, E: int, V: int, max_len: int) -> Population:
    pop = synth.small_random_population(seed, E, V, max_len=max_len, binary=ALL_BINARY,
                                        unary=ALL_UNARY)
    edge = Population.from_lists(_edge_expressions(V))
    from symbolic_regression_gpu_b200.population import concat
    return concat([edge, pop])


def _save(name: str, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


def eval_fixture():
    rng = np.random.default_rng(101)
    V, N = 3, 257
    X = _edge_dataset(rng, V, N)
    X[V] = rng.uniform(-2, 2, N).astype(np.float32)
    pop = _population_all_ops(102, 120, V, 40)
    pred = oracle.ref_predict(pop, X)
    mse, _ = oracle.ref_mse(pop, X, threads=4)
    _save("eval_all_ops.npz", tokens=pop.tokens, values=pop.values, offsets=pop.offsets, X=X,
          pred=pred, mse=mse)


def eval_workload_fixture():
    """Workload operators with EXP in place of the exp-clamp extension
    (which the reference does not have)."""
    rng = np.random.default_rng(201)
    V, N = 5, 1000
    X = rng.uniform(-3, 3, size=(V + 1, N)).astype(np.float32)
    unary = [op.EXP if u == op.EXP_CLAMP else u for u in op.WORKLOAD_UNARY]
    pop = synth.small_random_population(202, 200, V, max_len=63, binary=op.WORKLOAD_BINARY,
                                        unary=unary)
    mse, _ = oracle.ref_mse(pop, X, threads=4)
    sub = pop.slice(0, 40)
    pred = oracle.ref_predict(sub, X[:, :300].copy())
    _save("eval_workload_ops.npz", tokens=pop.tokens, values=pop.values, offsets=pop.offsets,
          X=X, mse=mse, pred_E=np.int64(40), pred_N=np.int64(300), pred=pred)


def _exp_clamp_dataset(rng, V: int, N: int) -> np.ndarray:
    """Arguments around the clamp (80), the float overflow of exp (88.72...)
    and beyond (100, 1e30, inf), NaN, and large negative ones."""
    X = rng.uniform(-3, 3, size=(V + 1, N)).astype(np.float32)
    around = np.array([79.0, 79.99999, 80.0, 80.00001, 80.5, 81.0, 88.0, 88.7, 88.72, 88.7228,
                       88.73, 89.0, 100.0, 1e30, np.inf, np.nan, -80.0, -87.3, -103.9, -104.0,
                       -120.0, -np.inf, 0.0, -0.0, 1e-40, 40.0, 44.35, 45.0], np.float32)
    k = min(N, around.size)
    for v in range(V):
        X[v, 3 * v:3 * v + k] = np.roll(around, 5 * v)[:k]
    X[V] = rng.uniform(-2, 2, N).astype(np.float32)
    return X


def _exp_clamp_expressions():
    C, X, EC = op.TOK_CONST, op.TOK_VAR, op.EXP_CLAMP
    return [
        ([EC, X], [0.0, 0.0]),
        ([EC, X], [0.0, 1.0]),
        ([EC, op.MUL, C, X], [0.0, 0.0, 30.0, 2.0]),          # 30 x: arguments up to +-90
        ([EC, op.NEG, X], [0.0, 0.0, 0.0]),
        ([EC, EC, X], [0.0, 0.0, 0.0]),                       # clamp of a clamped exp
        ([op.ADD, EC, X, EC, X], [0.0, 0.0, 0.0, 0.0, 1.0]),   # 2 e^80 stays finite
        ([op.MUL, EC, X, EC, X], [0.0, 0.0, 0.0, 0.0, 1.0]),   # e^160 overflows
        ([op.SUB, EC, X, EC, X], [0.0, 0.0, 0.0, 0.0, 0.0]),
        ([op.LOOSE_LOG, EC, X], [0.0, 0.0, 0.0]),
        ([op.LOOSE_DIV, C, EC, X], [0.0, 1.0, 0.0, 1.0]),
        ([EC, op.LOOSE_DIV, X, C], [0.0, 0.0, 0.0, 0.0125]),  # x / 0.0125: 80 at x = 1
        ([EC, C], [0.0, 80.0]),
        ([EC, C], [0.0, 88.7228]),
        ([EC, C], [0.0, 100.0]),
        ([op.EXP, X], [0.0, 0.0]),                            # the unclamped reference EXP
    ]


def eval_exp_clamp_fixture():
    """Opcode 32 at arguments around 80, 88.7 and 100 (edge expressions) and
    the workload operators with opcode 32 itself (random expressions), from
    the reference evaluator with the added case."""
    rng = np.random.default_rng(501)
    V, N = 3, 300
    X = _exp_clamp_dataset(rng, V, N)
    edge = Population.from_lists(_exp_clamp_expressions())
    pred = oracle.refx_predict(edge, X)
    mse, _ = oracle.refx_mse(edge, X, threads=4)
    rng = np.random.default_rng(502)
    V2, N2 = 5, 1000
    X2 = rng.uniform(-3, 3, size=(V2 + 1, N2)).astype(np.float32)
    X2[0, :40] = rng.uniform(20, 95, 40).astype(np.float32)   # large exp arguments
    pop = synth.small_random_population(503, 200, V2, max_len=63, binary=op.WORKLOAD_BINARY,
                                        unary=op.WORKLOAD_UNARY)
    mse2, _ = oracle.refx_mse(pop, X2, threads=4)
    sub = pop.slice(0, 60)
    pred2 = oracle.refx_predict(sub, X2[:, :400].copy())
    _save("eval_exp_clamp.npz", tokens=edge.tokens, values=edge.values, offsets=edge.offsets,
          X=X, pred=pred, mse=mse, w_tokens=pop.tokens, w_values=pop.values,
          w_offsets=pop.offsets, w_X=X2, w_mse=mse2, w_pred_E=np.int64(60),
          w_pred_N=np.int64(400), w_pred=pred2)


def hash_fixture():
    pop = _population_all_ops(301, 60, 4, 50)
    keys_ref, keys_gpu_path, sizes_ref, merkle_ref = [], [], [], []
    for t, v in pop:
        s, h = oracle.ref_merkle(t, v)
        sizes_ref.append(s)
        merkle_ref.append(h)
        for i in range(t.size):
            n = int(s[i])
            keys_ref.append(oracle.ref_flat_key(t[i:i + n], v[i:i + n]))
            keys_gpu_path.append(oracle.ref_flat_key_gpu_path(t[i:i + n], v[i:i + n]))
    _save("hash_kat.npz", tokens=pop.tokens, values=pop.values, offsets=pop.offsets,
          sizes=np.concatenate(sizes_ref), merkle=np.concatenate(merkle_ref),
          flat_keys=np.array(keys_ref, np.uint64),
          flat_keys_gpu_path=np.array(keys_gpu_path, np.uint64))


def detect_fixture():
    w = synth.cache_workload(seed=401, E=600, N=16, parents=40, shared=12)
    pop = w.population
    stats, groups, hints = oracle.ref_detect(pop, 3, 10)
    # A cache holding every detected key, slots in the reference's group order.
    keys = groups["key"]
    slots = np.arange(keys.size, dtype=np.int32)
    mark = oracle.ref_mark_cached(pop, keys, slots)
    # A cache holding a subset (every other key), as after a capacity limit.
    mark_half = oracle.ref_mark_cached(pop, keys[::2], slots[::2])
    _save("detect.npz", tokens=pop.tokens, values=pop.values, offsets=pop.offsets,
          num_subtrees=np.int64(stats["num_subtrees"]),
          avg_subtree_size=np.float64(stats["avg_subtree_size"]),
          coverage=np.float64(stats["coverage"]),
          covered_tokens=np.int64(stats["covered_tokens"]),
          group_size=groups["size"], group_count=groups["count"], group_key=groups["key"],
          hints=hints, mark_keys=keys, mark_slots=slots, mark_hints=mark,
          mark_half_hints=mark_half)


def main():
    if not (oracle.reference_available() and oracle.reference_expc_available()):
        sys.exit("oracle/_ref/libref_oracle.so or libref_expc.so is missing: run "
                 "`make -C oracle REF=<reference tree> ref` first")
    only = set(sys.argv[1:])
    if only:
        for name in only:
            globals()[name]()
        return
    eval_fixture()
    eval_workload_fixture()
    eval_exp_clamp_fixture()
    hash_fixture()
    detect_fixture()


if __name__ == "__main__":
    main()
