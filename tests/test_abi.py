"""The C-ABI library loads and exports every symbol its headers declare."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "symbolic_regression_gpu_b200", "lib", "libsr_eval.so")


def _declared_c_functions():
    src = open(os.path.join(ROOT, "include", "sr_eval.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sr_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_c_symbol():
    lib = ctypes.CDLL(LIB)
    names = _declared_c_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_declares_every_c_symbol():
    from symbolic_regression_gpu_b200 import _lib
    assert set(_declared_c_functions()) <= set(_lib._SIGNATURES)


@pytest.mark.skipif(shutil.which("nm") is None, reason="nm not available")
def test_reference_cpp_entry_points_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", LIB], capture_output=True,
                         text=True, check=True).stdout
    for sig in [
        "create_gpu_context()",
        "destroy_gpu_context(void*)",
        "evaluate_gpu_mse_wrapper(InputInfo&, float***, std::vector<float, "
        "std::allocator<float> >&, void*, bool, bool, RunStats&)",
        "create_gpu_simple_context()",
        "destroy_gpu_simple_context(void*)",
        "evaluate_gpu_simple_wrapper(InputInfo&, float***, std::vector<float, "
        "std::allocator<float> >&, void*, bool, RunStats&)",
    ]:
        assert sig in out, sig


def test_abi_version_and_status_strings():
    from symbolic_regression_gpu_b200 import _lib
    assert _lib.lib.sr_abi_version() == 2
    for s in range(13):
        assert _lib.status_string(s) not in ("", "unknown status")


def test_create_without_device_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from symbolic_regression_gpu_b200 import Evaluator, SrError, _lib
    with pytest.raises(SrError) as ei:
        Evaluator()
    assert ei.value.status == _lib.SR_ERR_NO_DEVICE


def test_launch_shape_options_are_checked_before_the_device():
    """Warps per block: 1..31, above 16 only at 8 datapoints per thread (or a
    tuned datapoint count, which then becomes 8).  The options are checked
    before the device is looked up, so this runs without a GPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import ctypes
    from symbolic_regression_gpu_b200 import _lib

    def create(dpt, warps):
        o = _lib.sr_options()
        assert _lib.lib.sr_options_init(ctypes.byref(o)) == _lib.SR_OK
        o.dpt, o.warps_per_block = dpt, warps
        ctx = ctypes.c_void_p()
        return _lib.lib.sr_create(ctypes.byref(o), ctypes.byref(ctx))

    for dpt, warps in [(8, 31), (0, 31), (8, 15), (4, 16), (16, 16), (0, 0)]:
        assert create(dpt, warps) == _lib.SR_ERR_NO_DEVICE, (dpt, warps)
    for dpt, warps in [(8, 32), (4, 17), (16, 31), (12, 8), (8, -1)]:
        assert create(dpt, warps) == _lib.SR_ERR_INVALID_ARGUMENT, (dpt, warps)


def test_null_arguments_are_rejected():
    from symbolic_regression_gpu_b200 import _lib
    assert _lib.lib.sr_create(None, None) == _lib.SR_ERR_INVALID_ARGUMENT
    assert _lib.lib.sr_options_init(None) == _lib.SR_ERR_INVALID_ARGUMENT
    assert _lib.lib.sr_destroy(None) == _lib.SR_OK
    assert _lib.lib.sr_launch(None) == _lib.SR_ERR_INVALID_ARGUMENT
