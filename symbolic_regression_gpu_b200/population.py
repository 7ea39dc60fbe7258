"""Populations in CSR form (the layout of the C ABI's sr_population).

Expression i is ``tokens[offsets[i]:offsets[i+1]]`` with the matching
``values`` (float64, as the reference InputInfo.values, src/utils/utils.h:31).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Iterable, List, Sequence, Tuple

import numpy as np


@dataclass
class Population:
    tokens: np.ndarray   # int32 [T]
    values: np.ndarray   # float64 [T]
    offsets: np.ndarray  # int64 [E+1]

    def __post_init__(self):
        self.tokens = np.ascontiguousarray(self.tokens, dtype=np.int32)
        self.values = np.ascontiguousarray(self.values, dtype=np.float64)
        self.offsets = np.ascontiguousarray(self.offsets, dtype=np.int64)
        if self.offsets.ndim != 1 or self.offsets.size < 1 or self.offsets[0] != 0:
            raise ValueError("offsets must be 1-D, start at 0")
        if self.tokens.shape != self.values.shape or self.tokens.size != self.offsets[-1]:
            raise ValueError("tokens/values/offsets sizes disagree")

    @classmethod
    def from_lists(cls, exprs: Iterable[Tuple[Sequence[int], Sequence[float]]]) -> "Population":
        toks: List[int] = []
        vals: List[float] = []
        offs = [0]
        for t, v in exprs:
            if len(t) != len(v):
                raise ValueError("tokens and values of an expression differ in length")
            toks.extend(int(x) for x in t)
            vals.extend(float(x) for x in v)
            offs.append(len(toks))
        return cls(np.array(toks, np.int32), np.array(vals, np.float64), np.array(offs, np.int64))

    @property
    def num_exprs(self) -> int:
        return int(self.offsets.size - 1)

    @property
    def num_tokens(self) -> int:
        return int(self.offsets[-1])

    def lengths(self) -> np.ndarray:
        return np.diff(self.offsets)

    def constant_counts(self) -> np.ndarray:
        """Constant tokens (TOK_CONST) per expression: the CSR row lengths of
        the gradient layout."""
        is_c = np.concatenate(([0], np.cumsum(self.tokens == 0, dtype=np.int64)))
        return np.diff(is_c[self.offsets])

    def expr(self, i: int) -> Tuple[np.ndarray, np.ndarray]:
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        return self.tokens[a:b], self.values[a:b]

    def __iter__(self):
        for i in range(self.num_exprs):
            yield self.expr(i)

    def subset(self, idx: Sequence[int]) -> "Population":
        return Population.from_lists(self.expr(int(i)) for i in idx)

    def slice(self, begin: int, end: int) -> "Population":
        a, b = int(self.offsets[begin]), int(self.offsets[end])
        return Population(self.tokens[a:b].copy(), self.values[a:b].copy(),
                          self.offsets[begin:end + 1] - a)

    def as_c(self):
        """sr_population view (the C ABI struct); the Population must outlive
        its use.  The library binding is imported here, not at module import,
        so that populations and the workload generators can be used where the
        library is not loaded (the bench's reference arm)."""
        from . import _lib
        p = _lib.sr_population()
        p.num_exprs = self.num_exprs
        p.tokens = self.tokens.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        p.values = self.values.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        p.offsets = self.offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        return p

    def constant_offsets(self) -> np.ndarray:
        """Exclusive prefix sum of per-expression constant counts (E+1)."""
        is_c = (self.tokens == 0).astype(np.int64)
        cs = np.concatenate([[0], np.cumsum(is_c)])
        return cs[self.offsets]

    def constants(self) -> np.ndarray:
        """Constant values (float32, as evaluated) in token order, CSR by constant_offsets."""
        return self.values[self.tokens == 0].astype(np.float32)

    def with_constants(self, consts: np.ndarray) -> "Population":
        vals = self.values.copy()
        vals[self.tokens == 0] = np.asarray(consts, dtype=np.float64)
        return Population(self.tokens.copy(), vals, self.offsets.copy())


def concat(pops: Sequence[Population]) -> Population:
    toks = np.concatenate([p.tokens for p in pops]) if pops else np.zeros(0, np.int32)
    vals = np.concatenate([p.values for p in pops]) if pops else np.zeros(0, np.float64)
    offs = [np.zeros(1, np.int64)]
    base = 0
    for p in pops:
        offs.append(p.offsets[1:] + base)
        base += p.num_tokens
    return Population(toks, vals, np.concatenate(offs))
