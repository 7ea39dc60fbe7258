"""Python host API over the C ABI: the population evaluator.

``Evaluator`` owns one ``sr_context``: a dataset resident on the GPU, the
compiled population, and the cross-generation subtree cache.  Every call goes
through libsr_eval.so; nothing here computes fitness itself.

Reference counterparts: evaluate_gpu_mse_wrapper (src/cleaned/cl_gpu_eval.cu:578-592,
subtree cache), evaluate_gpu_simple_wrapper (src/cleaned/cl_gpu_simple.cu:324-336).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from .population import Population

_F32P = ctypes.POINTER(ctypes.c_float)


def _f32ptr(a: np.ndarray):
    return a.ctypes.data_as(_F32P)


class Evaluator:
    """Population MSE evaluator on one GPU.

    Parameters mirror ``sr_options`` (include/sr_eval.h).  ``stream`` may be a
    ``torch.cuda.Stream`` (or a raw ``cudaStream_t`` integer); by default the
    library creates its own stream.
    """

    def __init__(self, device: int = -1, *, cache_capacity: int = 2048,
                 min_subtree_size: int = 3, min_subtree_freq: int = 10, dpt: int = 0,
                 warps_per_block: int = 0, autotune: bool = False, host_threads: int = 0,
                 tune_cache_path: Optional[str] = None, stream=None, use_graphs: bool = False,
                 device_detect: bool = False, smem_spill_slots: int = -1):
        opts = _lib.sr_options()
        _lib.check(_lib.lib.sr_options_init(ctypes.byref(opts)))
        self.device = device
        opts.device = device
        opts.cache_capacity = cache_capacity
        opts.min_subtree_size = min_subtree_size
        opts.min_subtree_freq = min_subtree_freq
        opts.dpt = dpt
        opts.warps_per_block = warps_per_block
        opts.autotune = 1 if autotune else 0
        opts.use_graphs = 1 if use_graphs else 0
        opts.device_detect = 1 if device_detect else 0
        opts.host_threads = host_threads
        opts.smem_spill_slots = smem_spill_slots
        self._tune_path = tune_cache_path.encode() if tune_cache_path else None
        opts.tune_cache_path = self._tune_path
        if stream is not None:
            opts.stream = ctypes.c_void_p(getattr(stream, "cuda_stream", stream))
        ctx = ctypes.c_void_p()
        _lib.check(_lib.lib.sr_create(ctypes.byref(opts), ctypes.byref(ctx)), what="sr_create")
        self._ctx = ctx
        self.stats = _lib.sr_stats()
        self.num_vars: Optional[int] = None
        self.num_dps: Optional[int] = None
        self._E = 0
        self._C = 0

    # ---- lifecycle -----------------------------------------------------
    def close(self):
        if getattr(self, "_ctx", None):
            # At interpreter shutdown the module globals may already be gone;
            # the process exit then releases the context with the device.
            lib = getattr(_lib, "lib", None) if _lib is not None else None
            if lib is not None:
                lib.sr_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int, what: str):
        _lib.check(status, self._ctx, what)

    @property
    def stream_handle(self) -> int:
        s = ctypes.c_void_p()
        self._check(_lib.lib.sr_get_stream(self._ctx, ctypes.byref(s)), "sr_get_stream")
        return s.value or 0

    def synchronize(self):
        self._check(_lib.lib.sr_synchronize(self._ctx), "sr_synchronize")

    # ---- dataset -------------------------------------------------------
    def set_data(self, X: np.ndarray):
        """X: [(V+1), N] float32 rows (column-major dataset), y in the last row."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        if X.ndim != 2 or X.shape[0] < 1:
            raise ValueError("X must be [(num_vars+1), num_dps]")
        V, N = X.shape[0] - 1, X.shape[1]
        self._check(_lib.lib.sr_set_data(self._ctx, _f32ptr(X), V, N), "sr_set_data")
        self.num_vars, self.num_dps = V, N

    def set_data_device(self, X, ld: Optional[int] = None):
        """X: a CUDA tensor [(V+1), N] float32 (row stride ld, default N)."""
        V, N = int(X.shape[0]) - 1, int(X.shape[1])
        ld = int(X.stride(0)) if ld is None else ld
        self._check(_lib.lib.sr_set_data_device(self._ctx, ctypes.c_void_p(X.data_ptr()), ld, V, N),
                    "sr_set_data_device")
        self.num_vars, self.num_dps = V, N

    # ---- evaluation ----------------------------------------------------
    @staticmethod
    def _flags(cache: bool, clear_cache: bool, plain: bool) -> int:
        f = 0
        if cache:
            f |= _lib.SR_EVAL_SUBTREE_CACHE
        if clear_cache:
            f |= _lib.SR_EVAL_CLEAR_CACHE
        if plain:
            f |= _lib.SR_EVAL_PLAIN
        return f

    def eval_mse(self, pop: Population, *, cache: bool = False, clear_cache: bool = False,
                 plain: bool = False) -> np.ndarray:
        """Per-expression MSE (float32 [E]); NaN where no datapoint is valid."""
        out = np.empty(pop.num_exprs, np.float32)
        cpop = pop.as_c()
        self._check(_lib.lib.sr_eval_mse(self._ctx, ctypes.byref(cpop),
                                         self._flags(cache, clear_cache, plain), _f32ptr(out),
                                         ctypes.byref(self.stats)), "sr_eval_mse")
        self._E = pop.num_exprs
        return out

    def eval_mse_fp64(self, pop: Population) -> np.ndarray:
        """FP64 reference MSE of every expression, evaluated on the GPU (the
        accuracy report of the FP32 results; float64 [E])."""
        out = np.empty(pop.num_exprs, np.float64)
        cpop = pop.as_c()
        self._check(_lib.lib.sr_eval_mse_fp64(self._ctx, ctypes.byref(cpop),
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                    "sr_eval_mse_fp64")
        return out

    def accuracy(self, pop: Population, mse: np.ndarray) -> np.ndarray:
        """|mse - mse_fp64| / |mse_fp64| per expression (NaN where either is
        not finite)."""
        ref = self.eval_mse_fp64(pop)
        m = np.asarray(mse, np.float64)
        with np.errstate(invalid="ignore", divide="ignore"):
            rel = np.abs(m - ref) / np.maximum(np.abs(ref), 1e-300)
        rel[~(np.isfinite(m) & np.isfinite(ref))] = np.nan
        return rel

    def prepare(self, pop: Population, *, cache: bool = False, clear_cache: bool = False,
                plain: bool = False, gradient: bool = False,
                grad_mode: int = _lib.SR_GRAD_CHECKPOINT):
        """Compile and upload `pop` for repeated launch().  gradient=True
        prepares the gradient launches (read_mse and read_grad); grad_mode is
        SR_GRAD_CHECKPOINT or SR_GRAD_RECOMPUTE, or-ed with
        SR_GRAD_REVERSE_ONLY to differentiate every expression in reverse
        mode."""
        cpop = pop.as_c()
        flags = self._flags(cache, clear_cache, plain)
        if gradient:
            flags = _lib.SR_EVAL_GRADIENT
            if (grad_mode & ~_lib.SR_GRAD_REVERSE_ONLY) == _lib.SR_GRAD_RECOMPUTE:
                flags |= _lib.SR_EVAL_GRAD_RECOMPUTE
            if grad_mode & _lib.SR_GRAD_REVERSE_ONLY:
                flags |= _lib.SR_EVAL_GRAD_REVERSE
        self._check(_lib.lib.sr_prepare(self._ctx, ctypes.byref(cpop), flags), "sr_prepare")
        self._E = pop.num_exprs
        self._C = int(np.count_nonzero(pop.tokens == 0))

    def launch(self):
        """Enqueue the prepared evaluation on the context stream (asynchronous)."""
        self._check(_lib.lib.sr_launch(self._ctx), "sr_launch")

    def read_mse(self) -> np.ndarray:
        out = np.empty(self._E, np.float32)
        self._check(_lib.lib.sr_read_mse(self._ctx, _f32ptr(out), ctypes.byref(self.stats)),
                    "sr_read_mse")
        return out

    def read_grad(self) -> np.ndarray:
        """d MSE / d constants of the last gradient launch (CSR over expressions)."""
        out = np.empty(max(self._C, 1), np.float32)
        self._check(_lib.lib.sr_read_grad(self._ctx, _f32ptr(out)), "sr_read_grad")
        return out[:self._C]

    def read_sums(self):
        """(FP64 sum of valid squared errors [E], valid count [E]) of the last
        launch: the partial result a datapoint shard contributes."""
        sums = np.empty(max(self._E, 1), np.float64)
        cnt = np.empty(max(self._E, 1), np.float64)
        P = ctypes.POINTER(ctypes.c_double)
        self._check(_lib.lib.sr_read_sums(self._ctx, sums.ctypes.data_as(P),
                                          cnt.ctypes.data_as(P)), "sr_read_sums")
        return sums[:self._E], cnt[:self._E]

    def read_grad_sums(self) -> np.ndarray:
        """FP64 sum over valid datapoints of d (squared error) / d constant, of
        the last gradient launch (CSR over expressions)."""
        out = np.empty(max(self._C, 1), np.float64)
        self._check(_lib.lib.sr_read_grad_sums(
            self._ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "sr_read_grad_sums")
        return out[:self._C]

    def eval_sums(self, pop: Population):
        """Batched evaluation of `pop` on this context's datapoints, returning
        read_sums() (the datapoint-shard contribution)."""
        self.eval_mse(pop)
        return self.read_sums()

    def last_launch_times(self):
        """(whole launch ms, main interpreter kernel ms) of the last launch."""
        a = ctypes.c_float()
        b = ctypes.c_float()
        self._check(_lib.lib.sr_last_launch_times(self._ctx, ctypes.byref(a), ctypes.byref(b)),
                    "sr_last_launch_times")
        return a.value, b.value

    def device_mse_ptr(self) -> int:
        p = ctypes.c_void_p()
        self._check(_lib.lib.sr_device_mse(self._ctx, ctypes.byref(p)), "sr_device_mse")
        return p.value or 0

    def predictions(self, pop: Population, dp_begin: int = 0,
                    dp_count: Optional[int] = None) -> np.ndarray:
        """Raw FP32 predictions [E, dp_count] (NaN/Inf included)."""
        if dp_count is None:
            dp_count = (self.num_dps or 0) - dp_begin
        out = np.empty((pop.num_exprs, dp_count), np.float32)
        cpop = pop.as_c()
        self._check(_lib.lib.sr_eval_predictions(self._ctx, ctypes.byref(cpop), dp_begin,
                                                 dp_count, _f32ptr(out)), "sr_eval_predictions")
        return out

    def eval_grad(self, pop: Population, mode: int = _lib.SR_GRAD_CHECKPOINT):
        """(mse [E], d mse / d constants [C]) with constants in token order."""
        nconst = int(np.count_nonzero(pop.tokens == 0))
        mse = np.empty(pop.num_exprs, np.float32)
        grad = np.empty(max(nconst, 1), np.float32)
        cpop = pop.as_c()
        self._check(_lib.lib.sr_eval_grad(self._ctx, ctypes.byref(cpop), mode, _f32ptr(mse),
                                          _f32ptr(grad), ctypes.byref(self.stats)),
                    "sr_eval_grad")
        self._E, self._C = pop.num_exprs, nconst
        return mse, grad[:nconst]

    def optimize_constants(self, pop: Population, steps: int = 20, lr: float = 0.05,
                           beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8,
                           mode: int = _lib.SR_GRAD_CHECKPOINT):
        """On-device Adam over every expression's constants.
        Returns (constants [C] after `steps`, mse [E] at those constants)."""
        nconst = int(np.count_nonzero(pop.tokens == 0))
        adam = _lib.sr_adam_options(steps, mode, lr, beta1, beta2, eps)
        consts = np.empty(max(nconst, 1), np.float32)
        mse = np.empty(pop.num_exprs, np.float32)
        cpop = pop.as_c()
        self._check(_lib.lib.sr_optimize_constants(self._ctx, ctypes.byref(cpop),
                                                   ctypes.byref(adam), _f32ptr(consts),
                                                   _f32ptr(mse), ctypes.byref(self.stats)),
                    "sr_optimize_constants")
        return consts[:nconst], mse

    def measure_pipes(self):
        """(FP32 FMA ops/s, MUFU ops/s, SM count) measured on this device."""
        f = ctypes.c_double()
        s = ctypes.c_double()
        n = ctypes.c_int32()
        self._check(_lib.lib.sr_measure_pipes(self._ctx, ctypes.byref(f), ctypes.byref(s),
                                              ctypes.byref(n)), "sr_measure_pipes")
        return f.value, s.value, n.value

    def measure_operator_rates(self, ops) -> dict:
        """{operator: evaluations/s} of each operator's FP32 semantics alone on
        this device (operator 0 = the measuring harness alone)."""
        arr = np.ascontiguousarray(list(ops), dtype=np.int32)
        out = np.zeros(max(arr.size, 1), np.float64)
        self._check(_lib.lib.sr_measure_operator_rates(
            self._ctx, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), int(arr.size),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "sr_measure_operator_rates")
        return {int(o): float(r) for o, r in zip(arr, out)}


def operator_bound_seconds(pop: Population, num_dps: int, rates: dict,
                           fp32_ops_per_s: float) -> float:
    """Accurate-operator bound of one evaluation of `pop`: every operator token
    at every datapoint costs 1 / rate of its operator less the harness's own
    cost (rates[0]), at least one FP32 instruction; leaves cost nothing."""
    toks = pop.tokens[pop.tokens > 0]
    ops, counts = np.unique(toks, return_counts=True)
    base = 1.0 / rates[0]
    per_dp = 0.0
    for o, c in zip(ops, counts):
        per_dp += c * max(1.0 / rates[int(o)] - base, 1.0 / fp32_ops_per_s)
    return per_dp * num_dps


# ---- host-only helpers (no GPU needed) ------------------------------------

def subtree_key(tokens, values) -> int:
    """Flat cache key of a token/value run (reference compute_subtree_hash_gpu,
    src/cleaned/cl_gpu_eval.cu:259-272)."""
    t = np.ascontiguousarray(tokens, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    return int(_lib.lib.sr_subtree_key(t.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                       v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), t.size))


def subtree_hashes(tokens, values):
    """(sizes int32 [L], Merkle hashes uint64 [L]) of one expression
    (reference detect.cpp:169-191)."""
    t = np.ascontiguousarray(tokens, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    sizes = np.empty(t.size, np.int32)
    hashes = np.empty(t.size, np.uint64)
    _lib.check(_lib.lib.sr_subtree_hashes(
        t.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
        v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), t.size,
        sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
        hashes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
    return sizes, hashes


def detect_subtrees(pop: Population, min_size: int = 3, min_freq: int = 10,
                    evaluator: Optional["Evaluator"] = None):
    """Common-subtree detection (reference detect_common_subtrees,
    src/utils/detect.cpp:120-387).  Returns (stats dict, groups dict of arrays).
    With an ``evaluator`` the detection runs on its GPU
    (sr_detect_subtrees_device), else on the host."""
    res = _lib.sr_detect_result()
    cpop = pop.as_c()
    if evaluator is not None:
        ctx = evaluator._ctx

        def call(*a):
            return _lib.lib.sr_detect_subtrees_device(ctx, *a)
    else:
        ctx = None
        call = _lib.lib.sr_detect_subtrees
    _lib.check(call(ctypes.byref(cpop), min_size, min_freq, 0, ctypes.byref(res), None, None,
                    None, None, None), ctx)
    n = res.num_subtrees
    ge = np.empty(max(n, 1), np.int32)
    gp = np.empty(max(n, 1), np.int32)
    gs = np.empty(max(n, 1), np.int32)
    gc = np.empty(max(n, 1), np.int32)
    gk = np.empty(max(n, 1), np.uint64)
    P = ctypes.POINTER
    _lib.check(call(
        ctypes.byref(cpop), min_size, min_freq, n, ctypes.byref(res),
        ge.ctypes.data_as(P(ctypes.c_int32)), gp.ctypes.data_as(P(ctypes.c_int32)),
        gs.ctypes.data_as(P(ctypes.c_int32)), gc.ctypes.data_as(P(ctypes.c_int32)),
        gk.ctypes.data_as(P(ctypes.c_uint64))), ctx)
    stats = {f: getattr(res, f) for f, _ in res._fields_ if f != "reserved0"}
    groups = {"expr": ge[:n], "pos": gp[:n], "size": gs[:n], "count": gc[:n], "key": gk[:n]}
    return stats, groups


def mark_cached(pop: Population, keys, slots) -> np.ndarray:
    """Cache-marking hints per token (reference mark_cached_subtrees_from_state,
    src/cleaned/cl_gpu_eval.cu:294-329)."""
    k = np.ascontiguousarray(keys, np.uint64)
    s = np.ascontiguousarray(slots, np.int32)
    hints = np.empty(max(pop.num_tokens, 1), np.int32)
    cpop = pop.as_c()
    P = ctypes.POINTER
    _lib.check(_lib.lib.sr_mark_cached(ctypes.byref(cpop), k.ctypes.data_as(P(ctypes.c_uint64)),
                                       s.ctypes.data_as(P(ctypes.c_int32)), k.size,
                                       hints.ctypes.data_as(P(ctypes.c_int32))))
    return hints[:pop.num_tokens]


def validate(pop: Population, num_vars: int):
    """(n_instr [E], spill_slots [E]); raises SrError naming the bad expression."""
    n_instr = np.empty(max(pop.num_exprs, 1), np.int32)
    slots = np.empty(max(pop.num_exprs, 1), np.int32)
    bad = ctypes.c_int32(-1)
    cpop = pop.as_c()
    P = ctypes.POINTER
    st = _lib.lib.sr_validate_population(ctypes.byref(cpop), num_vars,
                                         n_instr.ctypes.data_as(P(ctypes.c_int32)),
                                         slots.ctypes.data_as(P(ctypes.c_int32)),
                                         ctypes.byref(bad))
    if st != _lib.SR_OK:
        raise _lib.SrError(st, f"expression {bad.value}: {_lib.status_string(st)}")
    return n_instr[:pop.num_exprs], slots[:pop.num_exprs]


def compile_population(pop: Population, num_vars: int):
    """(bytecode uint32 [n_instr, 4], instruction offsets int64 [E+1],
    spill slots int32 [E]) exactly as the evaluator compiles the population."""
    P = ctypes.POINTER
    cpop = pop.as_c()
    offs = np.zeros(pop.num_exprs + 1, np.int64)
    slots = np.zeros(max(pop.num_exprs, 1), np.int32)
    _lib.check(_lib.lib.sr_compile_population(ctypes.byref(cpop), num_vars, None, 0,
                                              offs.ctypes.data_as(P(ctypes.c_int64)),
                                              slots.ctypes.data_as(P(ctypes.c_int32))))
    n = int(offs[-1])
    code = np.zeros((max(n, 1), 4), np.uint32)
    _lib.check(_lib.lib.sr_compile_population(ctypes.byref(cpop), num_vars,
                                              code.ctypes.data_as(P(ctypes.c_uint32)), n,
                                              offs.ctypes.data_as(P(ctypes.c_int64)),
                                              slots.ctypes.data_as(P(ctypes.c_int32))))
    return code[:n], offs, slots[:pop.num_exprs]
