"""Readers and writers of the reference's population and dataset files.

gen_N.txt (reference parse_input_info, src/utils/utils.cpp:122-233; written by
src/script/generate_evolution_data.py:124-134):
    <num_exprs>
    then per expression:
    <num_vars> <num_dps> <num_tokens>
    <tokens separated by spaces>
    <values separated by spaces>
    <data file name>

shared_data.txt (reference load_data_file, src/utils/utils.cpp:235-300): one
datapoint per line, num_vars+1 whitespace-separated numbers (x0 .. x_{V-1} y).

``load_shared_data`` / ``load_population`` are the fast paths: the library's
parallel loaders (sr_load_shared_data / sr_load_population, csrc/sr_io.cpp).
The ``read_*`` functions are the plain single-threaded readers.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Tuple

import numpy as np

from . import _lib
from .population import Population


def read_gen_file(path: str) -> Tuple[Population, List[int], List[int], List[str]]:
    """Returns (population, num_vars per expression, num_dps per expression,
    data file name per expression).  Numbers are read as whitespace-separated
    fields wherever they sit (the reference reads them with operator>>); after
    an expression's values one character is skipped and the rest of that line
    is the data file name (file.ignore() + getline in the reference)."""
    with open(path, "r") as f:
        text = f.read()
    pos = 0
    n_text = len(text)

    def field() -> str:
        nonlocal pos
        while pos < n_text and text[pos].isspace():
            pos += 1
        if pos >= n_text:
            raise ValueError(f"{path}: unexpected end of file")
        start = pos
        while pos < n_text and not text[pos].isspace():
            pos += 1
        return text[start:pos]

    n = int(field())
    if n <= 0:
        raise ValueError(f"{path}: invalid num_exprs {n}")
    exprs, nv, nd, files = [], [], [], []
    for _ in range(n):
        v, d, L = int(field()), int(field()), int(field())
        toks = [int(field()) for _ in range(L)]
        vals = [float(field()) for _ in range(L)]
        pos += 1  # file.ignore()
        end = text.find("\n", pos)
        end = n_text if end < 0 else end
        files.append(text[pos:end].strip())
        pos = end
        exprs.append((toks, vals))
        nv.append(v)
        nd.append(d)
    return Population.from_lists(exprs), nv, nd, files


def write_gen_file(path: str, pop: Population, num_vars: int, num_dps: int,
                   data_file: str) -> None:
    with open(path, "w") as f:
        f.write(f"{pop.num_exprs}\n")
        for t, v in pop:
            f.write(f"{num_vars} {num_dps} {t.size}\n")
            f.write(" ".join(str(int(x)) for x in t) + "\n")
            f.write(" ".join(repr(float(x)) for x in v) + "\n")
            f.write(f"{data_file}\n")


def read_shared_data(path: str, num_vars: int, num_dps: Optional[int] = None) -> np.ndarray:
    """[(num_vars+1), num_dps] float64 (the reference parses doubles with strtod
    and the evolution loop narrows them to float)."""
    flat = np.fromfile(path, sep=" ", dtype=np.float64)
    cols = num_vars + 1
    rows = flat.size // cols
    if num_dps is not None:
        if rows < num_dps:
            raise ValueError(f"{path}: {rows} datapoints, {num_dps} requested")
        rows = num_dps
    return np.ascontiguousarray(flat[: rows * cols].reshape(rows, cols).T)


def write_shared_data(path: str, X: np.ndarray, fmt: str = "%.9g") -> None:
    """X: [(V+1), N]; one datapoint per line.  The default format round-trips
    float32 values exactly."""
    np.savetxt(path, np.asarray(X).T, fmt=fmt, delimiter=" ")


def load_shared_data(path: str, num_vars: int, num_dps: Optional[int] = None,
                     threads: int = 0) -> np.ndarray:
    """[(num_vars+1), N] float32 through the parallel loader (values parsed as
    doubles and narrowed to float, as the reference loop does)."""
    n = ctypes.c_int64()
    bpath = os.fsencode(path)
    maxd = -1 if num_dps is None else int(num_dps)
    _lib.check(_lib.lib.sr_load_shared_data(bpath, num_vars, maxd, None, 0, ctypes.byref(n),
                                            threads), what=f"sr_load_shared_data({path})")
    N = n.value
    if num_dps is not None and N < num_dps:
        raise ValueError(f"{path}: {N} datapoints, {num_dps} requested")
    X = np.empty((num_vars + 1, max(N, 1)), np.float32)
    _lib.check(_lib.lib.sr_load_shared_data(bpath, num_vars, N,
                                            X.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                            X.shape[1], ctypes.byref(n), threads),
               what=f"sr_load_shared_data({path})")
    return X[:, :N]


def load_population(path: str, threads: int = 0):
    """(population, num_vars per expression, num_dps per expression, first
    data file name) through the parallel loader."""
    bpath = os.fsencode(path)
    E = ctypes.c_int32()
    T = ctypes.c_int64()
    _lib.check(_lib.lib.sr_load_population(bpath, ctypes.byref(E), ctypes.byref(T), None, None,
                                           None, None, None, None, 0, threads),
               what=f"sr_load_population({path})")
    tok = np.empty(max(T.value, 1), np.int32)
    val = np.empty(max(T.value, 1), np.float64)
    off = np.empty(E.value + 1, np.int64)
    nv = np.empty(E.value, np.int32)
    nd = np.empty(E.value, np.int32)
    name = ctypes.create_string_buffer(4096)
    P = ctypes.POINTER
    _lib.check(_lib.lib.sr_load_population(
        bpath, ctypes.byref(E), ctypes.byref(T), tok.ctypes.data_as(P(ctypes.c_int32)),
        val.ctypes.data_as(P(ctypes.c_double)), off.ctypes.data_as(P(ctypes.c_int64)),
        nv.ctypes.data_as(P(ctypes.c_int32)), nd.ctypes.data_as(P(ctypes.c_int32)), name,
        len(name), threads), what=f"sr_load_population({path})")
    pop = Population(tok[:T.value], val[:T.value], off)
    return pop, nv, nd, name.value.decode(errors="replace")
