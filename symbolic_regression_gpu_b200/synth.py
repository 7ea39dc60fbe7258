"""Seeded synthetic workloads in the reference's data model.

The reference measures on AI-Feynman data, which is not available here; these
generators stand in for it with seeded populations and datasets of the shapes,
sizes and value distributions of the five evaluation configurations:

  plain     1,000 ramped half-and-half expressions (depth 2-6), 3 variables,
            100k datapoints, x ~ U[1,5]
  batched   10,000 expressions, lengths 3-63 (geometric, mean 15), 5 variables,
            1M datapoints, x ~ U[-3,3]; 20 generations of subtree mutation /
            crossover
  cache     4,096 children of 256 parents sharing depth 2-4 subtrees,
            9 variables, 1M datapoints, x ~ U[0.5,10]
  grad      4,096 expressions with 1-8 constants, lengths 5-63, 4 variables,
            256k datapoints, x ~ U[1,5], target = hidden expression with
            perturbed constants
  large     100,000 expressions, lengths 3-127 (skewed, mean 25), 0-8
            constants, 10 variables, 4M datapoints, x ~ U[-5,5]

Operators: + - * protected-/ sin cos exp-clamped-at-80 protected-log|x|
sqrt|x| (opcodes.WORKLOAD_*).  Targets are y = hidden(x) + N(0, 0.01).
The tree operators (ramped half-and-half, subtree mutation, subtree
crossover) are the standard GP ones; the reference has its own versions in
src/utils/utils.cpp:995-1272.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import opcodes as op
from .population import Population

Expr = Tuple[List[int], List[float]]


@dataclass
class Workload:
    name: str
    population: Population
    X: np.ndarray                    # [(V+1), N] float32, y in the last row
    meta: Dict = field(default_factory=dict)

    @property
    def num_vars(self) -> int:
        return int(self.X.shape[0] - 1)

    @property
    def num_dps(self) -> int:
        return int(self.X.shape[1])


class TreeGen:
    """Random prefix-tree builder over an operator set."""

    def __init__(self, rng: np.random.Generator, num_vars: int,
                 binary: Sequence[int] = op.WORKLOAD_BINARY,
                 unary: Sequence[int] = op.WORKLOAD_UNARY,
                 const_range=(-5.0, 5.0), p_const: float = 0.3, p_unary: float = 0.35):
        self.rng = rng
        self.V = num_vars
        self.binary = list(binary)
        self.unary = list(unary)
        self.lo, self.hi = const_range
        self.p_const = p_const
        self.p_unary = p_unary

    def leaf(self, t: List[int], v: List[float]):
        if self.V == 0 or self.rng.random() < self.p_const:
            t.append(op.TOK_CONST)
            v.append(float(np.float32(self.rng.uniform(self.lo, self.hi))))
        else:
            t.append(op.TOK_VAR)
            v.append(float(self.rng.integers(self.V)))

    def depth_tree(self, depth: int, full: bool, t=None, v=None) -> Expr:
        """Full or grow tree of maximum depth `depth` (ramped half-and-half)."""
        t = [] if t is None else t
        v = [] if v is None else v
        if depth <= 0 or (not full and self.rng.random() < 0.3):
            self.leaf(t, v)
            return t, v
        if self.rng.random() < self.p_unary:
            t.append(int(self.rng.choice(self.unary)))
            v.append(0.0)
            self.depth_tree(depth - 1, full, t, v)
        else:
            t.append(int(self.rng.choice(self.binary)))
            v.append(0.0)
            self.depth_tree(depth - 1, full, t, v)
            self.depth_tree(depth - 1, full, t, v)
        return t, v

    def sized_tree(self, size: int, t=None, v=None) -> Expr:
        """Random tree with exactly `size` tokens."""
        t = [] if t is None else t
        v = [] if v is None else v
        if size <= 1:
            self.leaf(t, v)
        elif size == 2 or (size > 3 and self.rng.random() < self.p_unary * 0.6):
            t.append(int(self.rng.choice(self.unary)))
            v.append(0.0)
            self.sized_tree(size - 1, t, v)
        else:
            t.append(int(self.rng.choice(self.binary)))
            v.append(0.0)
            left = int(self.rng.integers(1, size - 1))
            self.sized_tree(left, t, v)
            self.sized_tree(size - 1 - left, t, v)
        return t, v


def subtree_sizes(tokens: Sequence[int]) -> List[int]:
    n = len(tokens)
    sizes = [1] * n
    for i in range(n - 1, -1, -1):
        tk = tokens[i]
        if tk <= 0:
            continue
        ar = 2 if tk < 10 else 1
        s, pos = 1, i + 1
        for _ in range(ar):
            if pos >= n:
                break
            s += sizes[pos]
            pos += sizes[pos]
        sizes[i] = s
    return sizes


def mutate(gen: TreeGen, e: Expr, max_tokens: int, min_tokens: int = 1,
           size_fair: bool = False) -> Expr:
    """Subtree mutation: a random subtree is replaced by a fresh random tree
    (size-fair: of a size within +-2 of the replaced one)."""
    t, v = e
    sizes = subtree_sizes(t)
    i = int(gen.rng.integers(len(t)))
    room = max_tokens - (len(t) - sizes[i])
    if room < 1:
        return list(t), list(v)
    if size_fair:
        lo, hi = max(1, sizes[i] - 2), min(room, sizes[i] + 2)
        new_size = int(gen.rng.integers(lo, max(lo, hi) + 1))
    else:
        new_size = int(gen.rng.integers(1, min(room, 2 * sizes[i] + 2) + 1))
    nt, nv = gen.sized_tree(new_size)
    ct = t[:i] + nt + t[i + sizes[i]:]
    if len(ct) < min_tokens:
        return list(t), list(v)
    return ct, v[:i] + nv + v[i + sizes[i]:]


def crossover(rng: np.random.Generator, a: Expr, b: Expr, max_tokens: int,
              min_tokens: int = 1, size_fair: bool = False) -> Expr:
    """Subtree crossover: a random subtree of `a` is replaced by a random
    subtree of `b` (up to 32 attempts to respect the length bounds; size-fair:
    the donor has between half and twice (+1) the replaced subtree's size)."""
    ta, va = a
    tb, vb = b
    sa, sb = subtree_sizes(ta), subtree_sizes(tb)
    i = int(rng.integers(len(ta)))
    for _ in range(min(len(tb), 32)):
        j = int(rng.integers(len(tb)))
        n = len(ta) - sa[i] + sb[j]
        if size_fair and not (sa[i] // 2 <= sb[j] <= 2 * sa[i] + 1):
            continue
        if min_tokens <= n <= max_tokens:
            return (ta[:i] + tb[j:j + sb[j]] + ta[i + sa[i]:],
                    va[:i] + vb[j:j + sb[j]] + va[i + sa[i]:])
    return list(ta), list(va)


def evolve(gen: TreeGen, pop: List[Expr], generations: int, max_tokens: int,
           min_tokens: int = 1, p_mutation: float = 0.2, elite_frac: float = 0.05,
           size_fair: bool = False) -> List[Expr]:
    """Fitness-free breeding: random parents, elites carried over, 20%
    subtree mutation / 80% subtree crossover."""
    rng = gen.rng
    n = len(pop)
    for _ in range(generations):
        n_elite = max(1, int(n * elite_frac))
        nxt = [pop[k] for k in rng.choice(n, n_elite, replace=False)]
        while len(nxt) < n:
            a = pop[int(rng.integers(n))]
            if rng.random() < p_mutation:
                nxt.append(mutate(gen, a, max_tokens, min_tokens, size_fair))
            else:
                b = pop[int(rng.integers(n))]
                nxt.append(crossover(rng, a, b, max_tokens, min_tokens, size_fair))
        pop = nxt
    return pop


# ---- targets -----------------------------------------------------------------

def _np_op(tok: int, a, b=None):
    with np.errstate(all="ignore"):
        if tok == op.ADD:
            return a + b
        if tok == op.SUB:
            return a - b
        if tok == op.MUL:
            return a * b
        if tok == op.LOOSE_DIV:
            d = np.where(np.abs(b) <= 1e-9, np.where(b < 0, -1e-9, 1e-9), b)
            return a / d
        if tok == op.SIN:
            return np.sin(a)
        if tok == op.COS:
            return np.cos(a)
        if tok == op.EXP_CLAMP:
            return np.exp(np.minimum(a, 80.0))
        if tok == op.LOOSE_LOG:
            return np.where(a == 0, -1e9, np.log(np.abs(np.where(a == 0, 1.0, a))))
        if tok == op.LOOSE_SQRT:
            return np.sqrt(np.abs(a))
    raise ValueError(f"target generator does not handle token {tok}")


def eval_target(expr: Expr, X: np.ndarray) -> np.ndarray:
    """Evaluate a (workload-operator) expression in float64 over X[:V] —
    used only to synthesise y."""
    t, v = expr
    stack = []
    for tk, vl in zip(reversed(t), reversed(v)):
        if tk == op.TOK_CONST:
            stack.append(np.full(X.shape[1], float(np.float32(vl))))
        elif tk == op.TOK_VAR:
            stack.append(X[int(vl)].astype(np.float64))
        elif 1 <= tk <= 9:
            a = stack.pop()
            b = stack.pop()
            stack.append(_np_op(tk, a, b))
        else:
            stack.append(_np_op(tk, stack.pop()))
    return stack[0]


def _target(rng: np.random.Generator, X: np.ndarray, gen: TreeGen, depth: int,
            hidden: Optional[Expr] = None) -> Tuple[np.ndarray, Expr]:
    for _ in range(200):
        h = hidden if hidden is not None else gen.depth_tree(depth, full=False)
        if hidden is None and len(h[0]) < 2 * depth + 1:
            continue
        yv = eval_target(h, X)
        varied = X.shape[1] < 2 or np.std(yv) > 1e-6
        if np.all(np.isfinite(yv)) and varied and np.max(np.abs(yv)) < 1e6:
            noise = rng.normal(0.0, 0.01, X.shape[1])
            return (yv + noise).astype(np.float32), h
        hidden = None
    raise RuntimeError("could not draw a finite hidden target")


def _dataset(rng, V: int, N: int, lo: float, hi: float) -> np.ndarray:
    X = np.empty((V + 1, N), np.float32)
    X[:V] = rng.uniform(lo, hi, size=(V, N)).astype(np.float32)
    return X


def _geometric_lengths(rng, n: int, lo: int, hi: int, mean: float) -> np.ndarray:
    p = 1.0 / max(mean - lo + 1.0, 1.0)
    out = lo + rng.geometric(p, size=n) - 1
    bad = out > hi
    while bad.any():
        out[bad] = lo + rng.geometric(p, size=int(bad.sum())) - 1
        bad = out > hi
    return out


def _set_constant_count(gen: TreeGen, e: Expr, lo: int, hi: int) -> Expr:
    """Turn variables into constants (or back) until lo <= #constants <= hi."""
    t, v = list(e[0]), list(e[1])
    consts = [i for i, tk in enumerate(t) if tk == op.TOK_CONST]
    varsx = [i for i, tk in enumerate(t) if tk == op.TOK_VAR]
    rng = gen.rng
    want = int(rng.integers(lo, hi + 1))
    want = min(want, len(consts) + len(varsx))
    while len(consts) > want and consts:
        i = consts.pop(int(rng.integers(len(consts))))
        t[i] = op.TOK_VAR
        v[i] = float(rng.integers(max(gen.V, 1)))
        varsx.append(i)
    while len(consts) < want and varsx:
        i = varsx.pop(int(rng.integers(len(varsx))))
        t[i] = op.TOK_CONST
        v[i] = float(np.float32(rng.uniform(gen.lo, gen.hi)))
        consts.append(i)
    return t, v


def repeat_stats(pop: Population, min_size: int = 3) -> Dict[str, float]:
    """Fraction of subtree occurrences (>= min_size tokens) whose token/value
    run occurs more than once in the population, and fraction of distinct such
    runs that occur more than once."""
    seen: Dict[Tuple, int] = {}
    total = 0
    for t, v in pop:
        tl, vl = t.tolist(), v.tolist()
        sizes = subtree_sizes(tl)
        for i, s in enumerate(sizes):
            if s >= min_size:
                key = (tuple(tl[i:i + s]), tuple(vl[i:i + s]))
                seen[key] = seen.get(key, 0) + 1
                total += 1
    repeated = sum(c for c in seen.values() if c > 1)
    distinct_rep = sum(1 for c in seen.values() if c > 1)
    return {"subtrees": total, "repeated_fraction": repeated / max(total, 1),
            "distinct": len(seen), "distinct_repeated_fraction": distinct_rep / max(len(seen), 1)}


def _length_meta(pop: Population) -> Dict[str, float]:
    L = pop.lengths()
    return {"E": pop.num_exprs, "tokens": int(L.sum()), "len_mean": float(L.mean()),
            "len_min": int(L.min()), "len_max": int(L.max())}


# ---- the five configurations ------------------------------------------------

def plain_workload(seed: int = 1, E: int = 1000, N: int = 100_000) -> Workload:
    rng = np.random.default_rng(seed)
    V = 3
    gen = TreeGen(rng, V)
    exprs = []
    depths = list(range(2, 7))
    for i in range(E):
        d = depths[(i // 2) % len(depths)]
        exprs.append(gen.depth_tree(d, full=(i % 2 == 0)))
    X = _dataset(rng, V, N, 1.0, 5.0)
    X[V], hidden = _target(rng, X, gen, 5)
    pop = Population.from_lists(exprs)
    meta = {"seed": seed, "V": V, "N": N, "x_range": [1, 5], **_length_meta(pop),
            "hidden": op.format_formula(*hidden)}
    return Workload("plain", pop, X, meta)


def batched_workload(seed: int = 2, E: int = 10_000, N: int = 1_000_000,
                     generations: int = 20) -> Workload:
    rng = np.random.default_rng(seed)
    V = 5
    gen = TreeGen(rng, V)
    lengths = _geometric_lengths(rng, E, 3, 63, 15.0)
    exprs = [gen.sized_tree(int(L)) for L in lengths]
    exprs = evolve(gen, exprs, generations, max_tokens=63, min_tokens=3, p_mutation=0.35,
                   size_fair=True)
    X = _dataset(rng, V, N, -3.0, 3.0)
    X[V], hidden = _target(rng, X, gen, 5)
    pop = Population.from_lists(exprs)
    meta = {"seed": seed, "V": V, "N": N, "x_range": [-3, 3], "generations": generations,
            **_length_meta(pop), "hidden": op.format_formula(*hidden)}
    return Workload("batched", pop, X, meta)


def cache_workload(seed: int = 3, E: int = 4096, N: int = 1_000_000, parents: int = 256,
                   shared: int = 48) -> Workload:
    rng = np.random.default_rng(seed)
    V = 9
    gen = TreeGen(rng, V)
    pool = []
    while len(pool) < shared:
        s = gen.depth_tree(int(rng.integers(2, 5)), full=bool(rng.integers(2)))
        if len(s[0]) >= 3:
            pool.append(s)
    par = []
    for _ in range(parents):
        t, v = gen.depth_tree(int(rng.integers(3, 6)), full=False)
        for _ in range(int(rng.integers(1, 3))):  # plant shared subtrees
            sizes = subtree_sizes(t)
            i = int(rng.integers(len(t)))
            s = pool[int(rng.integers(len(pool)))]
            t = t[:i] + list(s[0]) + t[i + sizes[i]:]
            v = v[:i] + list(s[1]) + v[i + sizes[i]:]
        par.append((t, v))
    exprs = []
    for _ in range(E):
        a = par[int(rng.integers(parents))]
        r = rng.random()
        if r < 0.5:
            child = crossover(rng, a, par[int(rng.integers(parents))], max_tokens=63, min_tokens=3)
        elif r < 0.8:
            child = mutate(gen, a, max_tokens=63, min_tokens=3)
        else:
            sizes = subtree_sizes(a[0])
            i = int(rng.integers(len(a[0])))
            s = pool[int(rng.integers(len(pool)))]
            t = a[0][:i] + list(s[0]) + a[0][i + sizes[i]:]
            v = a[1][:i] + list(s[1]) + a[1][i + sizes[i]:]
            child = (t, v) if 3 <= len(t) <= 63 else (list(a[0]), list(a[1]))
        exprs.append(child)
    X = _dataset(rng, V, N, 0.5, 10.0)
    X[V], hidden = _target(rng, X, gen, 4)
    pop = Population.from_lists(exprs)
    meta = {"seed": seed, "V": V, "N": N, "x_range": [0.5, 10], "parents": parents,
            "shared_pool": shared, **_length_meta(pop), "hidden": op.format_formula(*hidden)}
    return Workload("cache", pop, X, meta)


def grad_workload(seed: int = 4, E: int = 4096, N: int = 262_144) -> Workload:
    rng = np.random.default_rng(seed)
    V = 4
    gen = TreeGen(rng, V, p_const=0.35)
    lengths = _geometric_lengths(rng, E, 5, 63, 18.0)
    exprs = [_set_constant_count(gen, gen.sized_tree(int(L)), 1, 8) for L in lengths]
    X = _dataset(rng, V, N, 1.0, 5.0)
    # Hidden target: one expression with constants, perturbed by ~10%.
    while True:
        h = _set_constant_count(gen, gen.depth_tree(4, full=False), 2, 4)
        if sum(1 for tk in h[0] if tk == op.TOK_CONST) >= 1 and len(h[0]) >= 5:
            break
    ht = list(h[0])
    hv = [float(np.float32(x * (1.0 + 0.1 * rng.standard_normal()))) if tk == op.TOK_CONST
          else x for tk, x in zip(h[0], h[1])]
    X[V], hidden = _target(rng, X, gen, 4, hidden=(ht, hv))
    # Seed a quarter of the population with the unperturbed hidden structure.
    for k in range(0, E, 4):
        exprs[k] = (list(h[0]), list(h[1]))
    pop = Population.from_lists(exprs)
    meta = {"seed": seed, "V": V, "N": N, "x_range": [1, 5], **_length_meta(pop),
            "constants": int(np.count_nonzero(pop.tokens == 0)),
            "hidden": op.format_formula(*hidden)}
    return Workload("grad", pop, X, meta)


def large_workload(seed: int = 5, E: int = 100_000, N: int = 4_000_000) -> Workload:
    rng = np.random.default_rng(seed)
    V = 10
    gen = TreeGen(rng, V)
    # Skewed lengths in [3, 127] with mean ~25: geometric body.
    lengths = _geometric_lengths(rng, E, 3, 127, 25.0)
    exprs = [_set_constant_count(gen, gen.sized_tree(int(L)), 0, 8) for L in lengths]
    X = _dataset(rng, V, N, -5.0, 5.0)
    X[V], hidden = _target(rng, X, gen, 5)
    pop = Population.from_lists(exprs)
    meta = {"seed": seed, "V": V, "N": N, "x_range": [-5, 5], **_length_meta(pop),
            "constants": int(np.count_nonzero(pop.tokens == 0)),
            "hidden": op.format_formula(*hidden)}
    return Workload("large", pop, X, meta)


WORKLOADS = {
    "plain": plain_workload,
    "batched": batched_workload,
    "cache": cache_workload,
    "grad": grad_workload,
    "large": large_workload,
}


def small_random_population(seed: int, E: int, V: int, max_len: int = 31,
                            binary: Sequence[int] = op.WORKLOAD_BINARY,
                            unary: Sequence[int] = op.WORKLOAD_UNARY) -> Population:
    """A small mixed population for parity tests."""
    rng = np.random.default_rng(seed)
    gen = TreeGen(rng, V, binary=binary, unary=unary)
    exprs = [gen.sized_tree(int(rng.integers(1, max_len + 1))) for _ in range(E)]
    return Population.from_lists(exprs)
