"""Host-side validation and bytecode compilation (no GPU)."""
import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import _lib
from symbolic_regression_gpu_b200 import opcodes as op
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.population import Population

C, X = op.TOK_CONST, op.TOK_VAR


def _one(tokens, values=None):
    values = [0.0] * len(tokens) if values is None else values
    return Population.from_lists([(tokens, values)])


@pytest.mark.parametrize("tokens,status", [
    ([op.ADD, X], _lib.SR_ERR_MALFORMED_EXPRESSION),          # underflow
    ([X, X], _lib.SR_ERR_MALFORMED_EXPRESSION),               # two results
    ([op.SIN], _lib.SR_ERR_MALFORMED_EXPRESSION),
    ([28, X], _lib.SR_ERR_BAD_TOKEN),                          # unknown unary code
    ([-2], _lib.SR_ERR_BAD_TOKEN),
    ([X] * 0 + [op.ADD] * 600 + [C] * 601, _lib.SR_ERR_EXPRESSION_TOO_LONG),
])
def test_rejects(tokens, status):
    with pytest.raises(sg.SrError) as ei:
        sg.validate(_one(tokens), 3)
    assert ei.value.status == status


def test_empty_expression_rejected():
    pop = Population(np.zeros(0, np.int32), np.zeros(0), np.array([0, 0], np.int64))
    with pytest.raises(sg.SrError) as ei:
        sg.validate(pop, 3)
    assert ei.value.status == _lib.SR_ERR_MALFORMED_EXPRESSION


def test_bad_expression_index_reported():
    pop = Population.from_lists([([X], [0.0]), ([op.ADD, X, X], [0, 0, 1]), ([op.MUL, X], [0, 0])])
    with pytest.raises(sg.SrError) as ei:
        sg.validate(pop, 2)
    assert "expression 2" in str(ei.value)


def test_instruction_count_is_operator_count():
    pop = synth.small_random_population(7, 300, 3, max_len=63)
    n_instr, slots = sg.validate(pop, 3)
    for i, (t, _) in enumerate(pop):
        n_ops = int(np.count_nonzero(t > 0))
        assert n_instr[i] == max(n_ops, 1)


def test_spill_slots_bounded_by_tree_size():
    # Sethi-Ullman ordering: a tree needing k spill slots has >= 3*2^k - 1 tokens.
    pop = synth.small_random_population(8, 400, 3, max_len=127)
    _, slots = sg.validate(pop, 3)
    lens = pop.lengths()
    for k, L in zip(slots, lens):
        assert 3 * 2 ** int(k) - 1 <= max(L, 2)
    assert slots.max() <= 5


def test_balanced_tree_needs_log_slots():
    # ((x0+x1)*(x0+x1)) - ((x0+x1)*(x0+x1)) style full trees of sin-leaves.
    def full(depth):
        if depth == 0:
            return [op.SIN, X], [0.0, 0.0]
        a = full(depth - 1)
        b = full(depth - 1)
        return [op.ADD] + a[0] + b[0], [0.0] + a[1] + b[1]
    for d in range(1, 7):
        t, v = full(d)
        _, slots = sg.validate(Population.from_lists([(t, v)]), 1)
        assert slots[0] == d


def test_max_length_accepted():
    t = [op.ADD] * 511 + [X] * 512
    n_instr, slots = sg.validate(_one(t, [0.0] * 1023), 1)
    assert n_instr[0] == 511
