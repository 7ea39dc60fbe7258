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
    _U8 = POINTER(ctypes.c_uint8)
    lib.sro_error_bound.restype = None
    lib.sro_error_bound.argtypes = [c_int, _I32, _F64, _I64, c_int, c_int64, _F32, _F64, _F64,
                                    c_int, _F64, _F64, _U8, _F64, _F64, _I64, _I64, c_int]
    lib.sro_predict_f32_perturbed.restype = None
    lib.sro_predict_f32_perturbed.argtypes = [c_int, _I32, _F64, _I64, c_int, c_int64, _F32, _F64,
                                              c_uint64, c_int, _F32]
    return lib


_oracle = _load_oracle()
_ref = None
_refx = None
EXPC_PATH = os.path.join(HERE, "_ref", "libref_expc.so")


def reference_available() -> bool:
    return os.path.exists(REF_PATH)


def reference_expc_available() -> bool:
    return os.path.exists(EXPC_PATH)


def _refx_lib():
    """The reference's CPU evaluator with the one added case for opcode 32
    (oracle/ref_expc_shim.cpp)."""
    global _refx
    if _refx is None:
        if not reference_expc_available():
            raise FileNotFoundError(f"{EXPC_PATH} missing: run `make -C oracle REF=<reference "
                                    "tree> ref` where the reference tree exists")
        lib = ctypes.CDLL(EXPC_PATH)
        LL = POINTER(c_longlong)
        lib.refx_eval_single.restype = c_float
        lib.refx_eval_single.argtypes = [_I32, _F64, c_int, _F32, c_int]
        lib.refx_eval_mse.restype = c_double
        lib.refx_eval_mse.argtypes = [c_int, _I32, _F64, LL, c_int, c_int, _F32, _F32, c_int]
        lib.refx_predict.restype = None
        lib.refx_predict.argtypes = [c_int, _I32, _F64, LL, c_int, c_int, _F32, _F32, c_int]
        _refx = lib
    return _refx


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
        lib.ref_predict_all.restype = None
        lib.ref_predict_all.argtypes = [c_int, _I32, _F64, LL, c_int, c_int, _F32, _F32, c_int]
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


def ref_predict(pop, X: np.ndarray, threads: int = 0) -> np.ndarray:
    """Reference evaluate_single_expr at every datapoint [E, N]."""
    lib = _ref_lib()
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    out = np.empty((pop.num_exprs, N), np.float32)
    lib.ref_predict_all(pop.num_exprs, _p(t, _I32), _p(v, _F64),
                        o.ctypes.data_as(POINTER(c_longlong)), V, N, _p(X, _F32), _p(out, _F32),
                        threads or os.cpu_count())
    return out


def refx_mse(pop, X: np.ndarray, threads: int = 0):
    """The reference's evaluate_cpu_mse with opcode 32 added; (mse [E], ms)."""
    lib = _refx_lib()
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    out = np.empty(pop.num_exprs, np.float32)
    ms = lib.refx_eval_mse(pop.num_exprs, _p(t, _I32), _p(v, _F64),
                           o.ctypes.data_as(POINTER(c_longlong)), V, N, _p(X, _F32),
                           _p(out, _F32), threads or os.cpu_count())
    return out, ms


def refx_predict(pop, X: np.ndarray, threads: int = 0) -> np.ndarray:
    """The reference's evaluate_single_expr with opcode 32 added, [E, N]."""
    lib = _refx_lib()
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    out = np.empty((pop.num_exprs, N), np.float32)
    lib.refx_predict(pop.num_exprs, _p(t, _I32), _p(v, _F64),
                     o.ctypes.data_as(POINTER(c_longlong)), V, N, _p(X, _F32), _p(out, _F32),
                     threads or os.cpu_count())
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


# ---- the condition-aware parity rule ---------------------------------------------
#
# Maximum errors in ulps of the single-precision functions each side calls,
# per opcode (IEEE operators are correctly rounded on both sides and carry no
# entry).  Device: sin, cos and log are the library's own (csrc/sr_math.cuh),
# measured on every float argument of their fast paths against the correctly
# rounded value (tests/test_gpu_math.py: 1.57, 1.57 and 0.94 ulp; beyond the
# fast path sin / cos are CUDA's, documented at 2); the others are the CUDA
# Math API's documented maximum ulp errors over the full range (tanf 4,
# sinhf 3, coshf 2, tanhf 2, expf 2, asinf 2, acosf 2, atanf 2, powf 4).
# Host: glibc's float functions
# (the GNU C Library manual, "Known Maximum Errors in Math Functions", x86_64),
# taken as 1 ulp for sinf / cosf / expf / logf / powf and 2 for the others,
# at or above the listed figures.
def _ulp_table(per_op):
    a = np.zeros(64, np.float64)
    for k, u in per_op.items():
        a[k] = u
    return a


_DEV = {10: 2, 11: 2, 12: 4, 13: 3, 14: 2, 15: 2, 16: 2, 17: 1, 19: 2, 20: 2, 21: 2, 5: 4,
        9: 4, 22: 1, 32: 2}
_HOST = {10: 1, 11: 1, 12: 2, 13: 2, 14: 2, 15: 2, 16: 1, 17: 1, 19: 2, 20: 2, 21: 2, 5: 1,
         9: 1, 22: 1, 32: 1}
DEVICE_ULPS = _ulp_table(_DEV)
HOST_ULPS = _ulp_table(_HOST)

# Relative error of the device's reduction against the exact sum of the same
# squares (per lane FP32 Kahan summation over a tile's datapoints, 2 * 2^-24;
# FP64 beyond) plus the final float rounding of both MSEs (half an ulp each):
# the MSE allowance beyond the predictions' bound.
REDUCTION_REL = 2.5e-7
ULP_BAR = 4          # per-datapoint bar, ulps of the reference's value
MSE_BAR = 1e-6       # per-expression bar, relative to the reference's MSE
FP64_BAR = 1e-5      # accuracy bar against the FP64 evaluation


def error_bound(pop, X: np.ndarray, mode: int = 0, per_datapoint: bool = False,
                uA=None, uB=None, threads: int = 0) -> dict:
    """The running forward error bound of oracle/sr_oracle.c (sro_error_bound).

    mode 0: device FP32 against the reference's FP32 evaluation (centre =
    the reference's values, restated); mode 1: device FP32 against the exact
    value (centre = the FP64 evaluation).  Returns per expression ``mse``
    (the centre MSE in FP64), ``mse_bound``, ``flagged`` and ``valid``
    counts, and with per_datapoint [E, N] arrays ``pred``, ``bound`` and
    ``flag``."""
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    E = pop.num_exprs
    uA = DEVICE_ULPS if uA is None else np.ascontiguousarray(uA, np.float64)
    uB = HOST_ULPS if uB is None else np.ascontiguousarray(uB, np.float64)
    out = {"mse": np.empty(E, np.float64), "mse_bound": np.empty(E, np.float64),
           "flagged": np.empty(E, np.int64), "valid": np.empty(E, np.int64)}
    U8 = POINTER(ctypes.c_uint8)
    if per_datapoint:
        out["pred"] = np.empty((E, N), np.float64)
        out["bound"] = np.empty((E, N), np.float64)
        out["flag"] = np.empty((E, N), np.uint8)
        pp, pb, pf = _p(out["pred"], _F64), _p(out["bound"], _F64), out["flag"].ctypes.data_as(U8)
    else:
        pp = pb = None
        pf = None
    _oracle.sro_error_bound(E, _p(t, _I32), _p(v, _F64), _p(o, _I64), V, N, _p(X, _F32),
                            _p(uA, _F64), _p(uB, _F64), mode, pp, pb, pf,
                            _p(out["mse"], _F64), _p(out["mse_bound"], _F64),
                            _p(out["flagged"], _I64), _p(out["valid"], _I64),
                            threads or os.cpu_count())
    return out


def predict_f32_perturbed(pop, X: np.ndarray, k_ulps, seed: int = 0,
                          swap_sin_cos: bool = False) -> np.ndarray:
    """The float path with each transcendental result moved by up to
    k_ulps[op] ulps (tests of the bound); swap_sin_cos plants a mistake."""
    t, v, o = _pop_arrays(pop)
    X = np.ascontiguousarray(X, np.float32)
    V, N = X.shape[0] - 1, X.shape[1]
    k = np.ascontiguousarray(k_ulps, np.float64)
    out = np.empty((pop.num_exprs, N), np.float32)
    _oracle.sro_predict_f32_perturbed(pop.num_exprs, _p(t, _I32), _p(v, _F64), _p(o, _I64), V, N,
                                      _p(X, _F32), _p(k, _F64), seed, int(swap_sin_cos),
                                      _p(out, _F32))
    return out


def ulp32(x) -> np.ndarray:
    """Spacing of float32 numbers at |x| (the subnormal spacing below 2^-126)."""
    x = np.abs(np.asarray(x, np.float64))
    x = np.where(np.isfinite(x), np.minimum(x, 3.4028234663852886e38), 3.4028234663852886e38)
    _, e = np.frexp(x)
    return np.where(x < 1.1754943508222875e-38, 2.0 ** -149, np.ldexp(1.0, e - 24))


def datapoint_parity(pred_dev, pred_ref, bound, flag, ulp_bar: int = ULP_BAR) -> dict:
    """Per-datapoint rule: a flagged datapoint is exempt (discontinuity,
    singularity, overflow); every other one must agree on being finite and
    lie within max(ulp_bar ulps, bound) of the reference's value; it is
    exempt by conditioning when bound exceeds ulp_bar ulps (the expression
    amplifies the permitted per-operator differences past the bar)."""
    pd = np.asarray(pred_dev, np.float64)
    pr = np.asarray(pred_ref, np.float64)
    fl = np.asarray(flag).astype(bool)
    fin_d, fin_r = np.isfinite(pd), np.isfinite(pr)
    checked = ~fl
    bar = ulp_bar * ulp32(pr)
    cond = checked & fin_r & (bound > bar)
    both = checked & fin_r & fin_d
    with np.errstate(invalid="ignore"):
        diff = np.where(both, np.abs(pd - pr), 0.0)
    allow = np.maximum(bar, bound)
    finite_mismatch = checked & (fin_d != fin_r)
    nan_mismatch = checked & ~fin_r & ~fin_d & (np.isnan(pd) != np.isnan(pr))
    over = both & (diff > allow)
    inf_mismatch = checked & ~fin_r & ~fin_d & ~np.isnan(pr) & (pd != pr)
    n = int(pd.size)
    return {
        "datapoints": n,
        "exempt_flagged": int(fl.sum()),
        "exempt_conditioning": int(cond.sum()),
        "violations": int(over.sum() + finite_mismatch.sum() + nan_mismatch.sum() +
                          inf_mismatch.sum()),
        "within_bar": int((both & (diff <= bar)).sum()),
        "bit_identical": int((both & (pd == pr)).sum()),
        "max_excess_over_allowance": float(np.max(diff / np.maximum(allow, 1e-300)))
        if both.any() else 0.0,
    }


def mse_parity(mse_dev, mse_ref, mse_bound, flagged, bar: float = MSE_BAR,
               reduction_rel: float = REDUCTION_REL) -> dict:
    """Per-expression rule: an expression with a flagged datapoint is exempt;
    every other one must agree on NaN (no valid datapoint) and lie within
    max(bar, allowance) of the reference's MSE, allowance = the predictions'
    bound + reduction_rel * |MSE|; it is exempt by conditioning when the
    allowance exceeds the bar."""
    md = np.asarray(mse_dev, np.float64)
    mr = np.asarray(mse_ref, np.float64)
    fl = np.asarray(flagged) > 0
    checked = ~fl
    allow = np.asarray(mse_bound, np.float64) + reduction_rel * np.abs(mr)
    bar_abs = bar * np.abs(mr)
    fin = np.isfinite(mr) & np.isfinite(md)
    with np.errstate(invalid="ignore"):
        diff = np.where(fin, np.abs(md - mr), 0.0)
    nan_mismatch = checked & (np.isnan(md) != np.isnan(mr))
    inf_mismatch = checked & ~np.isnan(mr) & ~np.isnan(md) & (np.isinf(md) | np.isinf(mr)) & (md != mr)
    over = checked & fin & (diff > np.maximum(bar_abs, allow))
    cond = checked & fin & (allow > bar_abs)
    with np.errstate(invalid="ignore", divide="ignore"):
        rel = np.where(fin & (mr != 0), diff / np.abs(mr), 0.0)
    return {
        "expressions": int(md.size),
        "exempt_flagged": int(fl.sum()),
        "exempt_conditioning": int(cond.sum()),
        "violations": int(over.sum() + nan_mismatch.sum() + inf_mismatch.sum()),
        "nan_pattern_equal": bool((np.isnan(md) == np.isnan(mr)).all()),
        "within_bar_all": float(((rel <= bar) | ~fin).mean()) if md.size else 1.0,
        "within_bar_well_conditioned": float(((rel <= bar) | ~fin)[checked & ~cond].mean())
        if (checked & ~cond).any() else 1.0,
    }
