"""Index audit of the adjoint kernel (csrc/sr_adjoint.cu, adj_kernel) on the CPU.

Every shared/global index the kernel derives from a program — Jacobian-tape
entries (d out / d T at i - lo, d out / d b at db_base + kb), recompute-mode
segment entries and checkpoints, forward and adjoint spill slots, and the
constant accumulators (gacc[c * 32 + lane]) — is recomputed here from the
bytecode the library compiles, with the same formulas as the kernel and the
host planner (csrc/sr_capi_grad.cpp: tape_need, tape-length classes,
seg_cap, gmax), and asserted to lie inside the allocation the planner makes
for it.  Populations: the constant-optimisation workload, the large workload's
expressions (3-127 tokens), and deep random trees over every operator (long
programs with many segments and spill slots)."""
import numpy as np
import pytest

from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200 import opcodes as op
from symbolic_regression_gpu_b200.evaluator import compile_population
from symbolic_regression_gpu_b200.population import Population

K_SEG = 16                      # sr_adjoint.cu kSeg
MAX_ADJ_CONSTS = 64             # sr_capi_grad.cpp kMaxAdjConsts
TAPE_CLASSES = [8, 16, 32, 64, 128, 256, 512, 2048]
NO_CONST = 0x3FF
LEAF_C, B_S, B_C = 1, 1, 3
_LAST_MAX_TAPE = -1   # largest tape index of the last audited program


def _fields(w):
    return dict(op=w & 63, load=bool((w >> 6) & 1), lk=(w >> 7) & 3, bk=(w >> 9) & 7,
                spill=bool((w >> 12) & 1), slot=(w >> 13) & 31)


def _needs_db(bk):
    return bk in (B_C, B_S)


def _program_facts(code):
    """lo (lowest instruction holding a constant, len if none) and nb (db
    entries in [lo, len)), as the planner computes them."""
    n = len(code)
    lo = n
    for i, ins in enumerate(code):
        f = _fields(int(ins[0]))
        ca, cb = int(ins[3]) & 0x3FF, (int(ins[3]) >> 10) & 0x3FF
        if (f["load"] and f["lk"] == LEAF_C and ca != NO_CONST) or (f["bk"] == B_C and cb != NO_CONST):
            lo = i
            break
    nb = sum(1 for i in range(lo, n) if _needs_db(_fields(int(code[i][0]))["bk"]))
    return lo, nb


def _tape_need(n, lo, nb, smax, recompute):
    if recompute:
        nseg = (n + K_SEG - 1) // K_SEG
        return 2 * min(K_SEG, n) + smax + max(nseg - 1, 0) * (1 + smax)
    return (n - lo) + nb


def _audit_program(code, nconst, smax, tape_len, seg_cap, gmax, recompute):
    """Walks the kernel's index sequence of one program; returns the number
    of indices checked."""
    n = len(code)
    lo, _ = _program_facts(code)
    checked = 0
    global _LAST_MAX_TAPE
    _LAST_MAX_TAPE = -1

    def tape(idx):
        nonlocal checked
        global _LAST_MAX_TAPE
        assert 0 <= idx < tape_len, (idx, tape_len)
        _LAST_MAX_TAPE = max(_LAST_MAX_TAPE, idx)
        checked += 1

    def slot(s):
        nonlocal checked
        assert 0 <= s < max(smax, 1) and s < smax, (s, smax)
        checked += 1

    def const(c):
        nonlocal checked
        assert 0 <= c < nconst <= gmax, (c, nconst, gmax)
        checked += 1

    f_all = [_fields(int(ins[0])) for ins in code]
    last_seg = ((n - 1) // K_SEG) * K_SEG if recompute else 0
    t_lo = max(lo, last_seg) if recompute else lo
    db_base = seg_cap if recompute else n - lo
    ck_base = 2 * seg_cap + smax   # recompute: checkpoints after the adjoint slots

    def forward(i0, i1, tape_from, kb):
        for i in range(i0, i1):
            f = f_all[i]
            if recompute and i > 0 and i % K_SEG == 0 and i < last_seg and i + K_SEG > lo:
                ck = ck_base + (i // K_SEG - 1) * (1 + smax)
                for q in range(1 + smax):
                    tape(ck + q)
            if f["spill"]:
                slot(f["slot"])
            if f["load"] and f["lk"] == LEAF_C:
                ca = int(code[i][3]) & 0x3FF
                if ca != NO_CONST:
                    const(ca)
            if f["bk"] == B_S:
                slot(int(code[i][2]))
            if i >= tape_from:
                tape(i - (last_seg if recompute else lo))
                if _needs_db(f["bk"]):
                    tape(db_base + kb)
                    kb += 1
        return kb

    def backward(i_hi, i_lo, s0, kb):
        for i in range(i_hi - 1, i_lo - 1, -1):
            f = f_all[i]
            if _needs_db(f["bk"]):
                kb -= 1
                assert kb >= 0
            tape(i - s0)
            if _needs_db(f["bk"]):
                tape(db_base + kb)
                if f["bk"] == B_C:
                    cb = (int(code[i][3]) >> 10) & 0x3FF
                    if cb != NO_CONST:
                        const(cb)
                else:
                    slot(int(code[i][2]))          # adjoint slot of the spilled operand
            if f["load"]:
                if f["lk"] == LEAF_C and (int(code[i][3]) & 0x3FF) != NO_CONST:
                    const(int(code[i][3]) & 0x3FF)
                if f["spill"]:
                    slot(f["slot"])
        return kb

    if not recompute:
        kb = forward(0, n, t_lo, 0)
        kb = backward(n, lo, lo, kb)
        assert kb == 0
        return checked
    kb = forward(0, n, t_lo, 0)
    s0 = last_seg
    while s0 >= 0 and s0 + K_SEG > lo:
        s1 = min(n, s0 + K_SEG)
        if s0 != last_seg:
            if s0 > 0:
                ck = ck_base + (s0 // K_SEG - 1) * (1 + smax)
                for q in range(1 + smax):
                    tape(ck + q)
            kb = 0
            for i in range(s0, s1):
                f = f_all[i]
                if f["spill"]:
                    slot(f["slot"])
                if i >= lo:
                    tape(i - s0)
                    if _needs_db(f["bk"]):
                        tape(db_base + kb)
                        kb += 1
        kb = backward(s1, max(s0, lo), s0, kb)
        assert kb == 0
        s0 -= K_SEG
    return checked


def _audit(pop, num_vars):
    code, offs, slots = compile_population(pop, num_vars)
    smax = int(slots.max(initial=0))
    ncon = pop.constant_counts()
    E = pop.num_exprs
    total = 0
    for recompute in (False, True):
        needs, facts = [], []
        for x in range(E):
            c = code[offs[x]:offs[x + 1]]
            lo, nb = _program_facts(c)
            facts.append(c)
            needs.append(_tape_need(len(c), lo, nb, smax, recompute))
        # tape-length classes as the planner forms them
        klass = [min(next((k for k, t in enumerate(TAPE_CLASSES) if nd <= t),
                          len(TAPE_CLASSES) - 1), len(TAPE_CLASSES) - 1) for nd in needs]
        for k in set(klass):
            mem = [x for x in range(E) if klass[x] == k]
            tape_len = max(max(needs[x] for x in mem), 1)
            maxlen = max(max(len(facts[x]) for x in mem), 1)
            seg_cap = min(K_SEG, maxlen)
            gmax = max(max(int(ncon[x]) for x in mem), 1)
            for x in mem:
                total += _audit_program(facts[x], int(ncon[x]), smax, tape_len, seg_cap, gmax,
                                        recompute)
    return total


def test_adjoint_indices_constant_optimisation_workload():
    w = synth.grad_workload(seed=4, E=1500, N=64)
    assert _audit(w.population, w.num_vars) > 100_000


def test_adjoint_indices_large_workload_expressions():
    w = synth.large_workload(seed=5, E=1500, N=64)
    assert _audit(w.population, w.num_vars) > 100_000


def test_adjoint_indices_deep_trees_every_operator():
    rng = np.random.default_rng(31)
    gen = synth.TreeGen(rng, 3, p_const=0.4, binary=tuple(range(1, 10)),
                        unary=tuple(range(10, 28)) + (op.EXP_CLAMP,))
    exprs = [gen.depth_tree(int(d), full=bool(d % 2)) for d in rng.integers(2, 9, 300)]
    exprs += [gen.sized_tree(int(L)) for L in rng.integers(60, 400, 40)]
    pop = Population.from_lists(exprs)
    # expressions within the gradient path's constant limit (kMaxAdjConsts)
    keep = [i for i, c in enumerate(pop.constant_counts()) if c <= MAX_ADJ_CONSTS]
    assert _audit(pop.subset(keep), 3) > 50_000


def test_audit_catches_a_tape_one_entry_short():
    """A planted mistake (an allocation one entry shorter than the largest
    tape index the kernel uses) must fail the audit, in both modes; and the
    planner's tape_need covers that index."""
    w = synth.grad_workload(seed=4, E=200, N=64)
    code, offs, slots = compile_population(w.population, w.num_vars)
    smax = int(slots.max(initial=0))
    ncon = w.population.constant_counts()
    for recompute in (False, True):
        caught = 0
        for x in range(w.population.num_exprs):
            c = code[offs[x]:offs[x + 1]]
            lo, nb = _program_facts(c)
            need = _tape_need(len(c), lo, nb, smax, recompute)
            if int(ncon[x]) == 0:
                continue
            seg_cap = min(K_SEG, len(c))
            g = max(int(ncon[x]), 1)
            _audit_program(c, int(ncon[x]), smax, need, seg_cap, g, recompute)
            used = _LAST_MAX_TAPE + 1
            assert 1 <= used <= need
            with pytest.raises(AssertionError):
                _audit_program(c, int(ncon[x]), smax, used - 1, seg_cap, g, recompute)
            caught += 1
        assert caught > 50
