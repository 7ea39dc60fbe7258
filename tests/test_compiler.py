"""The bytecode compiler, verified on the CPU by emulation: executing the
compiled program must give bit-identical results to evaluating the prefix
tokens right to left with the same operator implementations."""
import sys

import numpy as np
import pytest

from emulate import run_bytecode, run_prefix
from symbolic_regression_gpu_b200 import opcodes as op
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.evaluator import compile_population
from symbolic_regression_gpu_b200.population import Population


def _same(a, b):
    return ((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all()


def _check_population(pop, X, V):
    code, offs, slots = compile_population(pop, V)
    for i, (t, v) in enumerate(pop):
        prog = code[offs[i]:offs[i + 1]]
        got = run_bytecode(prog, X, V)
        want = run_prefix(t, v, X, V)
        assert _same(got, want), f"expression {i}: {op.format_formula(t, v)}"


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_all_operators_random_trees(seed):
    rng = np.random.default_rng(seed)
    V = 3
    X = rng.uniform(-3, 3, size=(V + 1, 64)).astype(np.float32)
    X[0, :4] = [0.0, -0.0, 1e-12, 100.0]
    pop = synth.small_random_population(seed, 150, V, max_len=63,
                                        binary=op.BINARY_OPS, unary=op.UNARY_OPS)
    _check_population(pop, X, V)


def test_long_and_deep_trees():
    sys.setrecursionlimit(max(sys.getrecursionlimit(), 10_000))
    rng = np.random.default_rng(5)
    V = 2
    X = rng.uniform(-2, 2, size=(V + 1, 32)).astype(np.float32)
    gen = synth.TreeGen(rng, V)
    exprs = [gen.sized_tree(L) for L in (127, 255, 511, 1000, 1024)]

    def full(depth):  # perfectly balanced: needs `depth` spill slots
        if depth == 0:
            return [op.SIN, -1], [0.0, 1.0]
        a, b = full(depth - 1), full(depth - 1)
        return [op.SUB] + a[0] + b[0], [0.0] + a[1] + b[1]
    exprs.append(full(7))
    exprs.append(([op.ADD] * 511 + [-1] * 512, [0.0] * 511 + [0.0, 1.0] * 256))
    exprs.append(([op.SUB] * 100 + [0] + [op.SIN, -1] * 100,
                  [0.0] * 100 + [2.0] + [0.0, 1.0] * 100))   # right-deep chain
    pop = Population.from_lists(exprs)
    code, offs, slots = compile_population(pop, V)
    assert slots.max() <= 8
    assert slots[5] == 7
    _check_population(pop, X, V)


def test_out_of_range_variables_read_zero():
    X = np.arange(12, dtype=np.float32).reshape(3, 4)  # V = 2
    pop = Population.from_lists([([op.ADD, -1, -1], [0, 2.0, 0.0]),
                                 ([op.MUL, -1, -1], [0, 7.0, 1.0]),
                                 ([-1], [-1.0]), ([-1], [1.9])])
    _check_population(pop, X, 2)
    code, _, _ = compile_population(pop, 2)
    w = code[:, 0].astype(np.int64)
    leaf_kinds = set(((w[(w >> 6) & 1 == 1] >> 7) & 3).tolist())
    assert leaf_kinds == {0, 1}  # in-range variables and folded zeros


def test_leaves_are_folded_into_operators():
    pop = synth.small_random_population(9, 200, 4, max_len=40)
    code, offs, _ = compile_population(pop, 4)
    n_ops = np.array([max(int((t > 0).sum()), 1) for t, _ in pop])
    assert (np.diff(offs) == n_ops).all()


def test_reversed_opcodes_only_for_noncommutative():
    pop = synth.small_random_population(11, 300, 3, max_len=40, binary=op.BINARY_OPS,
                                        unary=op.UNARY_OPS)
    code, _, _ = compile_population(pop, 3)
    ops = set((code[:, 0].astype(np.int64) & 63).tolist())
    assert not (ops & {41, 43})            # ADD, MUL are never reversed
    assert ops & {42, 44, 45, 46, 47, 48, 49}
