"""The library's own sin, cos and log (csrc/sr_math.cuh) on every float
argument of their fast paths, against the correctly rounded value
(sr_check_math: the double-precision function rounded, errors in ulps of the
float result).  The bounds asserted here are the device column of the parity
rule's error table (oracle.DEVICE_ULPS): a change that makes a function less
accurate fails here before any parity test can be affected."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from symbolic_regression_gpu_b200 import _lib
from symbolic_regression_gpu_b200 import opcodes as op

pytestmark = pytest.mark.gpu


def _check(fn, begin, count):
    mx = ctypes.c_double()
    arg = ctypes.c_uint32()
    n, o5, o1 = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    st = _lib.lib.sr_check_math(fn, begin, count, ctypes.byref(mx), ctypes.byref(arg),
                                ctypes.byref(n), ctypes.byref(o5), ctypes.byref(o1))
    assert st == _lib.SR_OK, _lib.status_string(st)
    x = np.array([arg.value], np.uint32).view(np.float32)[0]
    return {"max_ulp": mx.value, "at": float(x), "checked": n.value,
            "over_half": o5.value, "over_one": o1.value}


def _both_signs(fn, hi_bits):
    """Every float in [0, hi] and [-hi, -0] (bit patterns 0..hi_bits)."""
    a = _check(fn, 0, hi_bits + 1)
    b = _check(fn, 0x80000000, hi_bits + 1)
    worst = a if a["max_ulp"] >= b["max_ulp"] else b
    return {"max_ulp": worst["max_ulp"], "at": worst["at"],
            "checked": a["checked"] + b["checked"],
            "over_half": a["over_half"] + b["over_half"],
            "over_one": a["over_one"] + b["over_one"]}


FAST_MAX_BITS = int(np.array([32768.0], np.float32).view(np.uint32)[0])


@pytest.mark.parametrize("name,fn,tok", [("sin", 10, op.SIN), ("cos", 11, op.COS)])
def test_sincos_every_argument_of_the_fast_path(name, fn, tok):
    r = _both_signs(fn, FAST_MAX_BITS)
    cuda = _both_signs(fn + 100, FAST_MAX_BITS)
    print(f"{name}: ours {r}, CUDA's {cuda}")
    assert r["checked"] > 2_000_000_000
    assert r["max_ulp"] <= oracle.DEVICE_ULPS[tok], r
    # also covers the loose variants that call them
    assert r["over_one"] <= cuda["over_one"] + r["checked"] // 10**6


def test_log_every_positive_argument():
    inf_bits = int(np.array([np.inf], np.float32).view(np.uint32)[0])
    r = _check(17, 0, inf_bits + 1)           # +0 .. +inf
    cuda = _check(117, 0, inf_bits + 1)
    print(f"log: ours {r}, CUDA's {cuda}")
    assert r["checked"] >= inf_bits
    assert r["max_ulp"] <= oracle.DEVICE_ULPS[op.LOG], r
    assert r["max_ulp"] <= oracle.DEVICE_ULPS[op.LOOSE_LOG], r


def test_special_values_of_log_and_sincos():
    neg = _check(17, 0x80000001, 0x7f800000 - 1)   # every negative finite: NaN
    assert neg["max_ulp"] == 0.0, neg
    big = _check(10, FAST_MAX_BITS + 1, 0x7f800000 - FAST_MAX_BITS)  # slow path: CUDA's sinf
    cuda = _check(110, FAST_MAX_BITS + 1, 0x7f800000 - FAST_MAX_BITS)
    assert big["max_ulp"] == cuda["max_ulp"]
