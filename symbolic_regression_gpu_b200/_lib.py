"""ctypes binding of libsr_eval.so (the C ABI declared in include/sr_eval.h).

The library is built in-tree by ``make -C symbolic_regression_gpu_b200/csrc``
(``__graft_entry__.build()`` does this).  There is no fallback: if the shared
library is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int32,
                    c_int64, c_uint32, c_uint64, c_void_p)

# SR_EVAL_LIBRARY selects another build of the library explicitly (a path that
# does not exist fails the import like a missing default build).
LIB_PATH = os.environ.get("SR_EVAL_LIBRARY") or os.path.join(
    os.path.dirname(os.path.abspath(__file__)), "lib", "libsr_eval.so")

# status codes (sr_status)
SR_OK = 0
SR_ERR_INVALID_ARGUMENT = 1
SR_ERR_BAD_TOKEN = 2
SR_ERR_MALFORMED_EXPRESSION = 3
SR_ERR_EXPRESSION_TOO_LONG = 4
SR_ERR_NO_DATA = 5
SR_ERR_CUDA = 6
SR_ERR_OUT_OF_MEMORY = 7
SR_ERR_DEVICE_TIMEOUT = 8
SR_ERR_DEVICE_CHECK = 9
SR_ERR_UNSUPPORTED = 10
SR_ERR_NO_DEVICE = 11
SR_ERR_TOO_MANY_VARS = 12

# evaluation flags
SR_EVAL_SUBTREE_CACHE = 0x1
SR_EVAL_CLEAR_CACHE = 0x2
SR_EVAL_PLAIN = 0x4
SR_EVAL_GRADIENT = 0x8
SR_EVAL_GRAD_RECOMPUTE = 0x10
SR_EVAL_GRAD_REVERSE = 0x20

# bounds of sr_eval_mse_device_noalloc (include/sr_eval.h)
SR_NOALLOC_SCRATCH_BYTES = 4 << 20
SR_NOALLOC_MAX_EXPRS = (SR_NOALLOC_SCRATCH_BYTES - 256) // 16

SR_GRAD_RECOMPUTE = 0
SR_GRAD_CHECKPOINT = 1
SR_GRAD_REVERSE_ONLY = 2


class sr_options(Structure):
    _fields_ = [
        ("device", c_int32),
        ("cache_capacity", c_int32),
        ("min_subtree_size", c_int32),
        ("min_subtree_freq", c_int32),
        ("dpt", c_int32),
        ("warps_per_block", c_int32),
        ("autotune", c_int32),
        ("use_graphs", c_int32),
        ("host_threads", c_int32),
        ("device_detect", c_int32),
        ("tune_cache_path", c_char_p),
        ("stream", c_void_p),
        ("smem_spill_slots", c_int32),
        ("reserved1", c_int32),
    ]


class sr_population(Structure):
    _fields_ = [
        ("num_exprs", c_int32),
        ("reserved0", c_int32),
        ("tokens", POINTER(c_int32)),
        ("values", POINTER(c_double)),
        ("offsets", POINTER(c_int64)),
    ]


class sr_stats(Structure):
    _fields_ = [
        ("total_eval_time_ms", c_double),
        ("detect_time_ms", c_double),
        ("data_transfer_time_ms", c_double),
        ("gpu_kernel_time_ms", c_double),
        ("num_subtrees", c_int32),
        ("new_subtrees", c_int32),
        ("avg_subtree_size", c_double),
        ("coverage", c_double),
        ("host_compile_time_ms", c_double),
        ("eval_kernel_time_ms", c_double),
        ("node_evals", c_int64),
        ("node_evals_executed", c_int64),
        ("kernel_launches", c_int32),
        ("cache_slots_used", c_int32),
        ("dpt", c_int32),
        ("warps_per_block", c_int32),
        ("blocks", c_int32),
        ("work_items", c_int32),
        ("declared_sfu_ops", c_double),
        ("declared_fp32_ops", c_double),
        ("h2d_bytes", c_int64),
        ("d2h_bytes", c_int64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class sr_detect_result(Structure):
    _fields_ = [
        ("num_subtrees", c_int32),
        ("reserved0", c_int32),
        ("total_tokens", c_int64),
        ("covered_tokens", c_int64),
        ("avg_subtree_size", c_double),
        ("coverage", c_double),
    ]


class sr_adam_options(Structure):
    _fields_ = [
        ("steps", c_int32),
        ("mode", c_int32),
        ("lr", c_float),
        ("beta1", c_float),
        ("beta2", c_float),
        ("eps", c_float),
    ]


SR_EVOLVE_MAX_STRIDE = 256


class sr_evolve_options(Structure):
    _fields_ = [
        ("num_vars", c_int32),
        ("max_tokens", c_int32),
        ("max_depth", c_int32),
        ("tournament", c_int32),
        ("const_min", c_float),
        ("const_max", c_float),
        ("prob_leaf", c_float),
        ("prob_const_leaf", c_float),
        ("prob_unary", c_float),
        ("elite_frac", c_float),
        ("mutation_prob", c_float),
        ("n_unary", c_int32),
        ("n_binary", c_int32),
        ("unary_ops", c_int32 * 32),
        ("binary_ops", c_int32 * 16),
        ("seed", c_uint64),
    ]


# Every symbol the header declares, with its ctypes signature.
_P = POINTER
_SIGNATURES = {
    "sr_abi_version": (c_int32, []),
    "sr_status_string": (c_char_p, [c_int32]),
    "sr_last_error": (c_char_p, [c_void_p]),
    "sr_options_init": (c_int32, [_P(sr_options)]),
    "sr_create": (c_int32, [_P(sr_options), _P(c_void_p)]),
    "sr_destroy": (c_int32, [c_void_p]),
    "sr_set_data": (c_int32, [c_void_p, _P(c_float), c_int32, c_int64]),
    "sr_set_data_rows": (c_int32, [c_void_p, _P(_P(c_float)), c_int32, c_int64]),
    "sr_set_data_device": (c_int32, [c_void_p, c_void_p, c_int64, c_int32, c_int64]),
    "sr_eval_mse": (c_int32, [c_void_p, _P(sr_population), c_uint32, _P(c_float), _P(sr_stats)]),
    "sr_prepare": (c_int32, [c_void_p, _P(sr_population), c_uint32]),
    "sr_launch": (c_int32, [c_void_p]),
    "sr_read_mse": (c_int32, [c_void_p, _P(c_float), _P(sr_stats)]),
    "sr_read_grad": (c_int32, [c_void_p, _P(c_float)]),
    "sr_inject_allocation_failure": (c_int32, [c_int64]),
    "sr_measure_operator_rates": (c_int32, [c_void_p, _P(c_int32), c_int32, _P(c_double)]),
    "sr_check_math": (c_int32, [c_int32, c_uint32, c_uint64, _P(c_double), _P(c_uint32),
                                _P(c_uint64), _P(c_uint64), _P(c_uint64)]),
    "sr_read_sums": (c_int32, [c_void_p, _P(c_double), _P(c_double)]),
    "sr_read_grad_sums": (c_int32, [c_void_p, _P(c_double)]),
    "sr_device_mse": (c_int32, [c_void_p, _P(c_void_p)]),
    "sr_last_launch_times": (c_int32, [c_void_p, _P(c_float), _P(c_float)]),
    "sr_eval_predictions": (c_int32, [c_void_p, _P(sr_population), c_int64, c_int64, _P(c_float)]),
    "sr_count_constants": (c_int32, [_P(sr_population), _P(c_int64)]),
    "sr_eval_grad": (c_int32, [c_void_p, _P(sr_population), c_int32, _P(c_float), _P(c_float),
                               _P(sr_stats)]),
    "sr_optimize_constants": (c_int32, [c_void_p, _P(sr_population), _P(sr_adam_options),
                                        _P(c_float), _P(c_float), _P(sr_stats)]),
    "sr_subtree_key": (c_uint64, [_P(c_int32), _P(c_double), c_int32]),
    "sr_subtree_hashes": (c_int32, [_P(c_int32), _P(c_double), c_int32, _P(c_int32), _P(c_uint64)]),
    "sr_detect_subtrees": (c_int32, [_P(sr_population), c_int32, c_int32, c_int32,
                                     _P(sr_detect_result), _P(c_int32), _P(c_int32), _P(c_int32),
                                     _P(c_int32), _P(c_uint64)]),
    "sr_detect_subtrees_device": (c_int32, [c_void_p, _P(sr_population), c_int32, c_int32,
                                            c_int32, _P(sr_detect_result), _P(c_int32),
                                            _P(c_int32), _P(c_int32), _P(c_int32), _P(c_uint64)]),
    "sr_mark_cached": (c_int32, [_P(sr_population), _P(c_uint64), _P(c_int32), c_int32,
                                 _P(c_int32)]),
    "sr_validate_population": (c_int32, [_P(sr_population), c_int32, _P(c_int32), _P(c_int32),
                                         _P(c_int32)]),
    "sr_compile_population": (c_int32, [_P(sr_population), c_int32, _P(c_uint32), c_int64,
                                        _P(c_int64), _P(c_int32)]),
    "sr_eval_mse_device_noalloc": (c_int32, [c_void_p, c_void_p, c_void_p, c_int32, c_void_p,
                                             c_int64, c_int32, c_int64, c_void_p, c_void_p]),
    "sr_eval_mse_fp64": (c_int32, [c_void_p, _P(sr_population), _P(c_double)]),
    "sr_evolve_options_init": (c_int32, [_P(sr_evolve_options), c_int32]),
    "sr_evolve_init": (c_int32, [c_void_p, _P(sr_evolve_options), c_int32, c_int32, c_void_p,
                                 c_void_p, c_void_p]),
    "sr_evolve_step": (c_int32, [c_void_p, _P(sr_evolve_options), c_int32, c_int32, c_int32,
                                 c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p]),
    "sr_prepare_device_population": (c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, c_int32,
                                               c_int32]),
    "sr_load_shared_data": (c_int32, [c_char_p, c_int32, c_int64, _P(c_float), c_int64,
                                      _P(c_int64), c_int32]),
    "sr_load_population": (c_int32, [c_char_p, _P(c_int32), _P(c_int64), _P(c_int32),
                                     _P(c_double), _P(c_int64), _P(c_int32), _P(c_int32),
                                     c_char_p, c_int32, c_int32]),
    "sr_get_stream": (c_int32, [c_void_p, _P(c_void_p)]),
    "sr_synchronize": (c_int32, [c_void_p]),
    "sr_measure_pipes": (c_int32, [c_void_p, _P(c_double), _P(c_double), _P(c_int32)]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C symbolic_regression_gpu_b200/csrc` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)  # AttributeError = the library lacks a declared symbol
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class SrError(RuntimeError):
    """A C-ABI call returned a status other than SR_OK."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"[{status}] {message}")


def status_string(status: int) -> str:
    return lib.sr_status_string(status).decode()


def check(status: int, ctx=None, what: str = "") -> None:
    if status != SR_OK:
        detail = lib.sr_last_error(ctx).decode() if ctx else ""
        msg = status_string(status)
        if what:
            msg = f"{what}: {msg}"
        if detail:
            msg = f"{msg} ({detail})"
        raise SrError(status, msg)
