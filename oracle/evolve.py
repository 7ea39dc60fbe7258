"""ORACLE — test infrastructure only.

Pure-Python restatement of the device-side generation loop
(symbolic_regression_gpu_b200/csrc/sr_evolve.cu), draw for draw, so that the
tests can check the device kernels bit for bit:

  * generation 0 and the subtree generator: reference generate_with_limit /
    build_node / emit_leaf, src/utils/utils.cpp:995-1108;
  * ranking: the reference's sort by fitness with NaN last,
    src/cleaned/cl_sr_system.cpp:286-290 (ties kept in index order);
  * breeding: elites, size-3 tournaments, 20 % subtree mutation
    (utils.cpp:1163-1204) / 80 % subtree crossover (utils.cpp:1206-1273),
    cl_sr_system.cpp:293-327.

The random numbers are the device's counter-based SplitMix64 stream per
(seed, generation, child), not the reference's std::mt19937 / rand()
sequence: same algorithm and distributions, different samples (the
distributions are compared with the reference's own generator in
tests/test_evolve_cpu.py).  Only tests/ import this module.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

M64 = (1 << 64) - 1
TOK_CONST, TOK_VAR = 0, -1


def mix64(z: int) -> int:
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


class Rng:
    """The device's per-child SplitMix64 stream (sr_evolve.cu, struct Rng)."""

    def __init__(self, seed: int, generation: int, child: int):
        ctr = ((generation & 0xFFFFFFFF) << 32) | (child & 0xFFFFFFFF)
        self.s = mix64((seed & M64) ^ mix64(ctr))

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        return mix64(self.s)

    def unit(self) -> np.float32:
        return np.float32((self.next() >> 40) * (1.0 / 16777216.0))

    def below(self, n: int) -> int:
        return ((self.next() >> 32) * n) >> 32

    def between(self, lo: int, hi: int) -> int:
        # reference rand_int: no draw when hi <= lo (utils.cpp:972-978)
        return lo if hi <= lo else lo + self.below(hi - lo + 1)

    def range(self, lo: float, hi: float) -> np.float32:
        lo32, hi32 = np.float32(lo), np.float32(hi)
        u = self.unit()
        return np.float32(lo32 + np.float32(np.float32(hi32 - lo32) * u))


def arity(t: int) -> int:
    if 1 <= t <= 9:
        return 2
    if 10 <= t <= 27 or t == 32:
        return 1
    return 0


def subtree_len(tok: Sequence[int], start: int) -> int:
    n = len(tok)
    if start < 0 or start >= n:
        return 0
    need, p = 1, start
    while need > 0 and p < n:
        need += arity(int(tok[p])) - 1
        p += 1
    return p - start


def default_options(num_vars: int) -> dict:
    """Reference EvolutionParams (src/utils/utils.h:178-187) and loop constants."""
    return dict(num_vars=num_vars, max_tokens=64, max_depth=5, tournament=3, const_min=-5.0,
                const_max=5.0, prob_leaf=0.1, prob_const_leaf=0.5, prob_unary=0.35,
                elite_frac=0.05, mutation_prob=0.2, unary_ops=list(range(10, 28)),
                binary_ops=list(range(1, 10)), seed=0x5EED5EED)


def generate(r: Rng, o: dict, limit: int, cap: int):
    """(tokens, values) of one generated subtree, or None when it would not
    fit in `cap` slots."""
    left = min(o["max_tokens"], limit)
    if left <= 0:
        return [], []
    f32 = np.float32
    tok: List[int] = []
    val: List[np.float32] = []
    nv = max(1, o["num_vars"])
    p_leaf, p_const, p_unary = f32(o["prob_leaf"]), f32(o["prob_const_leaf"]), f32(o["prob_unary"])
    U, B = o["unary_ops"], o["binary_ops"]

    def node(depth):
        nonlocal left
        must_leaf = depth >= o["max_depth"] or left == 1
        if not must_leaf and r.unit() < p_leaf:
            must_leaf = True
        if len(tok) >= cap:
            return -1
        if must_leaf:
            if r.unit() < p_const:
                tok.append(TOK_CONST)
                val.append(r.range(o["const_min"], o["const_max"]))
            else:
                tok.append(TOK_VAR)
                val.append(f32(r.between(0, nv - 1)))
            left -= 1
            return 0
        thresh = p_unary
        if left < 2:
            thresh = f32(0.0)
        if left < 3:
            thresh = f32(1.0)
        unary = r.unit() < thresh
        op = U[r.between(0, len(U) - 1)] if unary else B[r.between(0, len(B) - 1)]
        tok.append(op)
        val.append(f32(0.0))
        left -= 1
        return 1 if unary else 2

    a = node(0)
    if a < 0:
        return None
    frames = [[1, a]] if a > 0 else []
    while frames:
        if frames[-1][1] == 0:
            frames.pop()
            continue
        frames[-1][1] -= 1
        if left <= 0:
            if len(tok) >= cap:
                return None
            tok.append(TOK_VAR)
            val.append(f32(0.0))
            continue
        d = frames[-1][0]
        a = node(d)
        if a < 0:
            return None
        if a > 0:
            if len(frames) >= 64:
                return None
            frames.append([d + 1, a])
    if not tok:
        if cap < 1:
            return None
        tok, val = [TOK_CONST], [f32(0.0)]
    return tok, val


def evolve_init(o: dict, E: int, stride: int):
    out = []
    for i in range(E):
        g = generate(Rng(o["seed"], -1, i), o, o["max_tokens"], stride)
        out.append(g if g is not None else ([TOK_CONST], [np.float32(0.0)]))
    return out


def rank(fitness: np.ndarray) -> np.ndarray:
    f = np.asarray(fitness, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    keys = np.where(u & 0x80000000, (~u) & 0xFFFFFFFF, u | 0x80000000)
    keys = np.where(np.isnan(f), 0xFFFFFFFF, keys)
    return np.argsort(keys, kind="stable")


def evolve_step(o: dict, generation: int, pop: List[Tuple[list, list]], fitness: np.ndarray,
                stride: int):
    E = len(pop)
    order = rank(fitness)
    fit = np.asarray(fitness, np.float32)[order]
    elites = min(max(int(E * float(np.float32(o["elite_frac"]))), 1), E)
    mut_p = np.float32(o["mutation_prob"])
    children = []

    def tournament(r):
        best = r.below(E)
        for _ in range(o["tournament"] - 1):
            cand = r.below(E)
            if fit[cand] < fit[best]:
                best = cand
        return best

    for i in range(E):
        if i < elites:
            children.append(pop[order[i]])
            continue
        r = Rng(o["seed"], generation, i)
        at, av = pop[order[tournament(r)]]
        child = None
        if r.unit() < mut_p:
            n = len(at)
            if n > 0:
                idx = r.between(0, n - 1)
                old = subtree_len(at, idx) or 1
                max_new = o["max_tokens"] - (n - old)
                if max_new > 0:
                    tail = n - idx - old
                    g = generate(r, o, max_new, stride - idx - tail)
                    if g is not None:
                        child = (list(at[:idx]) + g[0] + list(at[idx + old:]),
                                 list(av[:idx]) + g[1] + list(av[idx + old:]))
        else:
            bt, bv = pop[order[tournament(r)]]
            if len(at) > 0 and len(bt) > 0:
                li = r.between(0, len(at) - 1)
                ls = subtree_len(at, li) or 1
                for _ in range(min(len(bt), 32)):
                    ri = r.between(0, len(bt) - 1)
                    rs = subtree_len(bt, ri)
                    if rs <= 0:
                        continue
                    total = len(at) - ls + rs
                    if total > o["max_tokens"] or total > stride:
                        continue
                    child = (list(at[:li]) + list(bt[ri:ri + rs]) + list(at[li + ls:]),
                             list(av[:li]) + list(bv[ri:ri + rs]) + list(av[li + ls:]))
                    break
        children.append(child if child is not None else (list(at), list(av)))
    return children


# ---- the reference's own GP operators (oracle/_ref, compiled unchanged) -------

def _ref_gp():
    import ctypes
    from ctypes import POINTER, c_float, c_int

    from . import oracle
    lib = oracle._ref_lib()
    if not getattr(lib, "_gp_ready", False):
        I, F = POINTER(c_int), POINTER(c_float)
        lib.ref_gp_seed.restype = None
        lib.ref_gp_seed.argtypes = [c_int]
        lib.ref_gp_generate.restype = c_int
        lib.ref_gp_generate.argtypes = [c_int, c_int, c_int, I, F, c_int]
        lib.ref_gp_mutate.restype = c_int
        lib.ref_gp_mutate.argtypes = [c_int, c_int, c_int, I, F, c_int, I, F, c_int]
        lib.ref_gp_crossover.restype = c_int
        lib.ref_gp_crossover.argtypes = [c_int, c_int, c_int, I, F, c_int, I, F, c_int, I, F,
                                         c_int]
        lib.ref_gp_subtree_size.restype = c_int
        lib.ref_gp_subtree_size.argtypes = [I, c_int, c_int]
        lib._gp_ready = True
    return lib


def _arrs(t, v):
    import ctypes
    ta = np.ascontiguousarray(t, np.int32)
    va = np.ascontiguousarray(v, np.float32)
    return ta, va, ta.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), \
        va.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def ref_seed(seed: int):
    _ref_gp().ref_gp_seed(seed)


def ref_generate(num_vars: int, max_tokens: int = 64, max_depth: int = 5, cap: int = 512):
    lib = _ref_gp()
    ot, ov, otp, ovp = _arrs(np.zeros(cap), np.zeros(cap))
    n = lib.ref_gp_generate(num_vars, max_tokens, max_depth, otp, ovp, cap)
    return list(ot[:n]), list(ov[:n])


def ref_mutate(parent, num_vars: int, max_tokens: int = 64, max_depth: int = 5, cap: int = 512):
    lib = _ref_gp()
    pt, pv, ptp, pvp = _arrs(*parent)
    ot, ov, otp, ovp = _arrs(np.zeros(cap), np.zeros(cap))
    n = lib.ref_gp_mutate(num_vars, max_tokens, max_depth, ptp, pvp, len(pt), otp, ovp, cap)
    return list(ot[:n]), list(ov[:n])


def ref_crossover(a, b, num_vars: int, max_tokens: int = 64, max_depth: int = 5, cap: int = 512):
    lib = _ref_gp()
    at, av, atp, avp = _arrs(*a)
    bt, bv, btp, bvp = _arrs(*b)
    ot, ov, otp, ovp = _arrs(np.zeros(cap), np.zeros(cap))
    n = lib.ref_gp_crossover(num_vars, max_tokens, max_depth, atp, avp, len(at), btp, bvp,
                             len(bt), otp, ovp, cap)
    return list(ot[:n]), list(ov[:n])


def ref_subtree_size(tok, start: int) -> int:
    t, _, tp, _ = _arrs(tok, np.zeros(len(tok)))
    return _ref_gp().ref_gp_subtree_size(tp, len(t), start)
