"""ORACLE — test infrastructure only.

ctypes binding of the CPU checker:
  * ``lib/libsr_oracle.so``  — the C restatement (oracle/sr_oracle.c);
  * ``_ref/libref_oracle.so`` — the reference's own CPU evaluator, subtree
    detection and cache marking compiled unchanged (built here from the
    reference tree; shipped prebuilt to other machines).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It is the checker, never the thing measured or shipped.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_int64, c_longlong, c_uint64

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_PATH = os.path.join(HERE, "lib", "libsr_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_oracle.so")

_I32 = POINTER(c_int32)
_F64 = POINTER(c_double)
_F32 = POINTER(c_float)
_I64 = POINTER(c_int64)
_U64 = POINTER(c_uint64)


def _p(a, t):
    return a.ctypes.data_as(t)


def _load_oracle():
    if not os.path.exists(ORACLE_PATH):
        raise ImportError(f"{ORACLE_PATH} missing: run `make -C oracle`")
    lib = ctypes.CDLL(ORACLE_PATH)
    lib.sro_op_f32.restype = c_float
    lib.sro_op_f32.argtypes = [c_int, c_float, c_float]
    lib.sro_op_f64.restype = c_double
    lib.sro_op_f64.argtypes = [c_int, c_double, c_double]
    lib.sro_eval_f32.restype = c_float
    lib.sro_eval_f32.argtypes = [_I32, _F64, c_int, _F32, c_int]
    lib.sro_predict_f32.restype = None
    lib.sro_predict_f32.argtypes = [c_int, _I32, _F64, _I64, c_int, c_int64, _F32, _F32, c_int]
    lib.sro_mse_f32.restype = None
    lib.sro_mse_f32.argtypes = [c_int, _I32, _F64, _I64, c_int, c_int64, _F32, _F32, c_int]
    lib.sro_mse_f64.restype = None
    lib.sro_mse_f64.argtypes = [c_int, _I32, _F64, _I64, c_int, c_int64, _F32, _F64, _I64, c_int]
    lib.sro_grad_f64.restype = None
    lib.sro_grad_f64.argtypes = [c_int, _I32, _F64, _I64, c_int, c_int64, _F32, _F64, _F64,
                                 _F64, c_int]
    lib.sro_flat_key.restype = c_uint64
    lib.sro_flat_key.argtypes = [_I32, _F64, c_int]
    lib.sro_merkle.restype = None
    lib.sro_merkle.argtypes = [_I32, _F64, c_int, _I32, _U64]
    return lib


_oracle = _load_oracle()
_ref = None


def reference_available() -> bool:
    return os.path.exists(REF_PATH)


def _ref_lib():
    global _ref
    if _ref is None:
        if not reference_available():
            raise FileNotFoundError(f"{REF_PATH} missing: run `make -C oracle ref` where the "
                                    "reference tree exists")
        lib = ctypes.CDLL(REF_PATH)
        LL = POINTER(c_longlong)
        lib.ref_eval_single.restype = c_float
        lib.ref_eval_single.argtypes = [_I32, _F64, c_int, _F32, c_int]
        lib.ref_eval_mse.restype = c_double
        lib.ref_eval_mse.argtypes = [c_int, _I32, _F64, LL, c_int, c_int, _F32, _F32, c_int]
        lib.ref_compute_hash.restype = c_uint64
        lib.ref_compute_hash.argtypes = [_I32, _F64, c_int]
        lib.ref_subtree_size.restype = c_int
        lib.ref_subtree_size.argtypes = [_I32, c_int, c_int]
        lib.ref_merkle.restype = None
        lib.ref_merkle.argtypes = [_I32, _F64, c_int, _I32, _U64]
        lib.ref_detect.restype = c_int
        lib.ref_detect.argtypes = [c_int, _I32, _F64, LL, c_int, c_int, c_int, _I32, _I32, _U64,
                                   _I32, _F64, _F64, LL]
        lib.ref_subtree_hash_gpu.restype = c_uint64
        lib.ref_subtree_hash_gpu.argtypes = [_I32, _F64, c_int]
        lib.ref_subtree_size_state.restype = c_int
        lib.ref_subtree_size_state.argtypes = [_I32, c_int, c_int]
        lib.ref_mark_cached.restype = None
        lib.ref_mark_cached.argtypes = [c_int, _I32, _F64, LL, _U64, _I32, c_int, _I32]
        _ref = lib
    return _ref


def _pop_arrays(pop):
    t = np.ascontiguousarray(pop.tokens, np.int32)
    v = np.ascontiguousarray(pop.values, np.float64)
    o = np.ascontiguousarray(pop.offsets, np.int64)
    return t, v, o


# ---- restatement ------------------------------------------------------------

def op_f32(op: int, a: float, b: float = 0.0) -> float:
    return _oracle.sro_op_f32(op, a, b)


def op_f64(op: int, a: float, b: float = 0.0) -> float:
    return _oracle.sro_op_f64(op, a, b)


def predict_f32(pop, X: np.ndarray, threads: int = 0) -> np.ndarray:
    """Per-datapoint FP32 predictions [E, N] (reference evaluate_single_expr semantics)."""
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    out = np.empty((pop.num_exprs, N), np.float32)
    _oracle.sro_predict_f32(pop.num_exprs, _p(t, _I32), _p(v, _F64), _p(o, _I64), V, N,
                            _p(X, _F32), _p(out, _F32), threads or os.cpu_count())
    return out


def mse_f32(pop, X: np.ndarray, threads: int = 0) -> np.ndarray:
    """Reference float-path MSE (reference evaluate_cpu_mse semantics)."""
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    out = np.empty(pop.num_exprs, np.float32)
    _oracle.sro_mse_f32(pop.num_exprs, _p(t, _I32), _p(v, _F64), _p(o, _I64), V, N,
                        _p(X, _F32), _p(out, _F32), threads or os.cpu_count())
    return out


def mse_f64(pop, X: np.ndarray, threads: int = 0):
    """(FP64 MSE [E], valid counts [E]): FP64 evaluation and accumulation."""
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    out = np.empty(pop.num_exprs, np.float64)
    cnt = np.empty(pop.num_exprs, np.int64)
    _oracle.sro_mse_f64(pop.num_exprs, _p(t, _I32), _p(v, _F64), _p(o, _I64), V, N,
                        _p(X, _F32), _p(out, _F64), _p(cnt, _I64), threads or os.cpu_count())
    return out, cnt


def grad_f64(pop, X: np.ndarray, threads: int = 0, with_abs: bool = False):
    """(FP64 MSE [E], FP64 d MSE / d constants [C], constants in token order);
    with_abs adds the mean absolute per-datapoint contribution [C]."""
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    mse = np.empty(pop.num_exprs, np.float64)
    C = int(np.count_nonzero(t == 0))
    grad = np.empty(max(C, 1), np.float64)
    gabs = np.empty(max(C, 1), np.float64) if with_abs else None
    _oracle.sro_grad_f64(pop.num_exprs, _p(t, _I32), _p(v, _F64), _p(o, _I64), V, N,
                         _p(X, _F32), _p(mse, _F64), _p(grad, _F64),
                         _p(gabs, _F64) if with_abs else None, threads or os.cpu_count())
    if with_abs:
        return mse, grad[:C], gabs[:C]
    return mse, grad[:C]


def mse_of_predictions(pred: np.ndarray, y: np.ndarray) -> np.ndarray:
    """FP64 MSE of given FP32 predictions [E, N] (the reduction-only reference):
    float difference and square as in the reference, FP64 sum."""
    y = np.asarray(y, np.float32)
    valid = np.isfinite(pred)
    d = (pred - y[None, :]).astype(np.float32)
    sq = np.where(valid, d * d, np.float32(0)).astype(np.float64)
    cnt = valid.sum(axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(cnt > 0, sq.sum(axis=1) / np.maximum(cnt, 1), np.nan)


def flat_key(tokens, values) -> int:
    t = np.ascontiguousarray(tokens, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    return int(_oracle.sro_flat_key(_p(t, _I32), _p(v, _F64), t.size))


def merkle(tokens, values):
    t = np.ascontiguousarray(tokens, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    s = np.empty(t.size, np.int32)
    h = np.empty(t.size, np.uint64)
    _oracle.sro_merkle(_p(t, _I32), _p(v, _F64), t.size, _p(s, _I32), _p(h, _U64))
    return s, h


# ---- the reference itself -----------------------------------------------------

def ref_mse(pop, X: np.ndarray, threads: int = 0):
    """Reference evaluate_cpu_mse; returns (mse [E], its own wall time in ms)."""
    lib = _ref_lib()
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    out = np.empty(pop.num_exprs, np.float32)
    ms = lib.ref_eval_mse(pop.num_exprs, _p(t, _I32), _p(v, _F64),
                          o.ctypes.data_as(POINTER(c_longlong)), V, N, _p(X, _F32), _p(out, _F32),
                          threads or os.cpu_count())
    return out, ms


def ref_predict(pop, X: np.ndarray) -> np.ndarray:
    """Reference evaluate_single_expr at every datapoint [E, N] (small inputs only)."""
    lib = _ref_lib()
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    rowsT = np.ascontiguousarray(X[:V].T)  # [N, V]
    out = np.empty((pop.num_exprs, N), np.float32)
    for e in range(pop.num_exprs):
        tk, vl = pop.expr(e)
        tk = np.ascontiguousarray(tk, np.int32)
        vl = np.ascontiguousarray(vl, np.float64)
        for dp in range(N):
            out[e, dp] = lib.ref_eval_single(_p(tk, _I32), _p(vl, _F64), tk.size,
                                             _p(rowsT[dp], _F32), V)
    return out


def ref_flat_key(tokens, values) -> int:
    t = np.ascontiguousarray(tokens, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    return int(_ref_lib().ref_compute_hash(_p(t, _I32), _p(v, _F64), t.size))


def ref_flat_key_gpu_path(tokens, values) -> int:
    t = np.ascontiguousarray(tokens, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    return int(_ref_lib().ref_subtree_hash_gpu(_p(t, _I32), _p(v, _F64), t.size))


def ref_merkle(tokens, values):
    t = np.ascontiguousarray(tokens, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    s = np.empty(t.size, np.int32)
    h = np.empty(t.size, np.uint64)
    _ref_lib().ref_merkle(_p(t, _I32), _p(v, _F64), t.size, _p(s, _I32), _p(h, _U64))
    return s, h


def ref_detect(pop, min_size: int = 3, min_freq: int = 10):
    """Reference detect_common_subtrees: (stats, groups with size/count/key, hints [T])."""
    lib = _ref_lib()
    t, v, o = _pop_arrays(pop)
    cap = max(1, pop.num_tokens)
    gs = np.empty(cap, np.int32)
    gc = np.empty(cap, np.int32)
    gk = np.empty(cap, np.uint64)
    hints = np.empty(max(1, pop.num_tokens), np.int32)
    avg = c_double()
    cov = c_double()
    covered = c_longlong()
    n = lib.ref_detect(pop.num_exprs, _p(t, _I32), _p(v, _F64),
                       o.ctypes.data_as(POINTER(c_longlong)), min_size, min_freq, cap,
                       _p(gs, _I32), _p(gc, _I32), _p(gk, _U64), _p(hints, _I32),
                       ctypes.byref(avg), ctypes.byref(cov), ctypes.byref(covered))
    stats = {"num_subtrees": n, "avg_subtree_size": avg.value, "coverage": cov.value,
             "covered_tokens": covered.value}
    return stats, {"size": gs[:n], "count": gc[:n], "key": gk[:n]}, hints[:pop.num_tokens]


def ref_mark_cached(pop, keys, slots) -> np.ndarray:
    lib = _ref_lib()
    t, v, o = _pop_arrays(pop)
    k = np.ascontiguousarray(keys, np.uint64)
    s = np.ascontiguousarray(slots, np.int32)
    hints = np.empty(max(1, pop.num_tokens), np.int32)
    lib.ref_mark_cached(pop.num_exprs, _p(t, _I32), _p(v, _F64),
                        o.ctypes.data_as(POINTER(c_longlong)), _p(k, _U64), _p(s, _I32), k.size,
                        _p(hints, _I32))
    return hints[:pop.num_tokens]
