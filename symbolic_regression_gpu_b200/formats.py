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
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np

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
