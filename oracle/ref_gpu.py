"""ORACLE — test infrastructure only.

The reference's own GPU evaluators, compiled unchanged for sm_100a into
oracle/_ref/libref_gpu.so (oracle/ref_gpu_run.cu, oracle/ref_gpu_run_simple.cu),
timed on a population: the bench's same-GPU comparison point.

  * simple:  evaluate_gpu_simple_wrapper (src/cleaned/cl_gpu_simple.cu:187-336):
             eval_simple_kernel writes every squared error to an [E x N] buffer,
             reduce_mse_kernel_simple sums it per expression;
  * subtree: evaluate_gpu_mse_wrapper (src/cleaned/cl_gpu_eval.cu:332-592): host
             subtree detection, cache update and skeleton rewrite, then
             eval_subtrees_kernel / eval_skeletons_kernel / reduce_mse_kernel,
             with the cache kept across calls (clear_cache false, as the
             reference's evolution loop calls it, cl_sr_system.cpp:207).

Run as its own process, ``python -m oracle.ref_gpu <in.npz> <out.json>
[--steps K]``, because the reference prints a timing breakdown to stdout on
every call and ends the process on any CUDA error.  Before any call the
population is checked against the limits of the reference kernels, which are
respected by construction:
  * int32 indexing (expr_idx * total_dps, cache_idx * total_dps): expressions
    run in chunks with E_chunk * N < 2^31, and the subtree path only when
    2048 * N < 2^31 (N < 1,048,576);
  * a 60-deep local stack (MAX_STACK_SIZE) and a 32-entry variable cache
    (MAX_NUM_FEATURES): every expression's stack depth <= 60, V + 1 <= 32,
    every variable index in [0, V) (the kernels read X at any other index);
  * opcode 32 (exp clamped at 80) is not a reference operator: it is run as
    the reference's EXP (16), the same expf call.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time
from ctypes import POINTER, c_double, c_float, c_int, c_longlong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GPU_PATH = os.path.join(HERE, "_ref", "libref_gpu.so")
MAX_STACK = 60
MAX_FEATURES = 32
INT32_LIMIT = 2 ** 31
CACHE_SLOTS = 2048


def available() -> bool:
    return os.path.exists(GPU_PATH)


def stack_depths(tokens: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """Largest stack depth of each expression's right-to-left evaluation."""
    step = np.where(tokens <= 0, 1, np.where(tokens < 10, -1, 0)).astype(np.int64)
    out = np.zeros(offsets.size - 1, np.int64)
    for e in range(offsets.size - 1):
        seg = step[offsets[e]:offsets[e + 1]][::-1]
        out[e] = int(np.cumsum(seg).max(initial=0))
    return out


def check_limits(tokens, values, offsets, V: int, N: int) -> str | None:
    """None when the population respects every limit above, else why not."""
    if V + 1 > MAX_FEATURES:
        return f"{V} variables: the reference kernels hold at most {MAX_FEATURES - 1}"
    var = tokens == -1
    vi = values[var].astype(np.int64)
    if var.any() and (vi.min() < 0 or vi.max() >= V):
        return "a variable index outside [0, V)"
    known = (tokens >= -1) & ((tokens <= 27) | (tokens == 32))
    if not known.all():
        return "a token outside the reference encoding"
    if stack_depths(tokens, offsets).max(initial=0) > MAX_STACK:
        return f"an expression deeper than the reference's {MAX_STACK}-entry stack"
    if N >= INT32_LIMIT:
        return "N >= 2^31"
    return None


def _lib():
    lib = ctypes.CDLL(GPU_PATH)
    I32, F64, F32 = POINTER(c_int), POINTER(c_double), POINTER(c_float)
    LL = POINTER(c_longlong)
    lib.refg_simple_create.restype = c_void_p
    lib.refg_simple_destroy.argtypes = [c_void_p]
    lib.refg_simple_eval.argtypes = [c_void_p, c_int, I32, F64, LL, c_int, c_int, F32, F32, c_int,
                                     F64]
    lib.refg_subtree_create.restype = c_void_p
    lib.refg_subtree_destroy.argtypes = [c_void_p]
    lib.refg_subtree_eval.argtypes = [c_void_p, c_int, I32, F64, LL, c_int, c_int, F32, F32, c_int,
                                      c_int, F64]
    return lib


class _Quiet:
    """Sends the reference's per-call stdout breakdown to /dev/null."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def run(tokens, values, offsets, X, steps: int = 2, paths=("simple", "subtree")) -> dict:
    tokens = np.ascontiguousarray(tokens, np.int32).copy()
    tokens[tokens == 32] = 16
    values = np.ascontiguousarray(values, np.float64)
    offsets = np.ascontiguousarray(offsets, np.int64)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    E = offsets.size - 1
    why = check_limits(tokens, values, offsets, V, N)
    if why:
        return {"unavailable": why}
    chunk = max(1, min(E, (INT32_LIMIT - 1) // max(N, 1)))
    bounds = list(range(0, E, chunk)) + [E]
    lib = _lib()
    I32, F64, F32 = POINTER(c_int), POINTER(c_double), POINTER(c_float)
    node_evals = int(offsets[-1]) * N
    res = {"exprs": E, "num_dps": N, "chunk_exprs": chunk, "chunks": len(bounds) - 1,
           "node_evals_per_generation": node_evals}
    mse = np.empty(E, np.float32)
    for path in paths:
        if path == "subtree" and CACHE_SLOTS * N >= INT32_LIMIT:
            res[path] = {"unavailable": "N >= 1,048,576 overflows the cache kernel's int32 index"}
            continue
        ctx = lib.refg_simple_create() if path == "simple" else lib.refg_subtree_create()
        first = True
        gens = []
        for g in range(steps + 1):
            wall = kern = xfer = detect = 0.0
            t0 = time.perf_counter()
            for a, b in zip(bounds[:-1], bounds[1:]):
                o = offsets[a:b + 1] - offsets[a]
                t = np.ascontiguousarray(tokens[offsets[a]:offsets[b]])
                v = np.ascontiguousarray(values[offsets[a]:offsets[b]])
                st = np.zeros(4, np.float64)
                out = np.empty(b - a, np.float32)
                args = (ctx, b - a, t.ctypes.data_as(I32), v.ctypes.data_as(F64),
                        o.ctypes.data_as(POINTER(c_longlong)), V, N, X.ctypes.data_as(F32),
                        out.ctypes.data_as(F32), int(first))
                with _Quiet():
                    if path == "simple":
                        lib.refg_simple_eval(*args, st.ctypes.data_as(F64))
                    else:
                        lib.refg_subtree_eval(*args, 0, st.ctypes.data_as(F64))
                first = False
                mse[a:b] = out
                wall += st[0]
                xfer += st[1]
                kern += st[2]
                detect += st[3]
            gens.append({"call_ms": wall, "kernel_ms": kern, "transfer_ms": xfer,
                         "detect_ms": detect, "host_wall_ms": (time.perf_counter() - t0) * 1e3})
        if path == "simple":
            lib.refg_simple_destroy(ctx)
        else:
            lib.refg_subtree_destroy(ctx)
        timed = gens[1:]
        kern = sum(x["kernel_ms"] for x in timed) / len(timed)
        call = sum(x["call_ms"] for x in timed) / len(timed)
        res[path] = {"kernel_ms": kern, "call_ms": call,
                     "kernel_node_evals_per_s": node_evals / (kern * 1e-3),
                     "call_node_evals_per_s": node_evals / (call * 1e-3),
                     "generations_timed": len(timed), "first_generation": gens[0],
                     "finite_mse": int(np.isfinite(mse).sum())}
        res[path + "_mse"] = mse.copy()
    return res


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("inp")
    ap.add_argument("out")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--paths", default="simple,subtree")
    a = ap.parse_args(argv)
    if not available():
        json.dump({"unavailable": f"{GPU_PATH} was not built"}, open(a.out, "w"))
        return 0
    d = np.load(a.inp)
    res = run(d["tokens"], d["values"], d["offsets"], d["X"], steps=a.steps,
              paths=tuple(a.paths.split(",")))
    mses = {k: res.pop(k) for k in list(res) if k.endswith("_mse")}
    if mses:
        np.savez(os.path.splitext(a.out)[0] + "_mse.npz", **mses)
    json.dump(res, open(a.out, "w"))
    return 0


if __name__ == "__main__":
    sys.exit(main())
