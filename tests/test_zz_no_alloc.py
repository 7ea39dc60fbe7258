"""The allocation-free entry point, sr_eval_mse_device_noalloc.

It serves callers that keep the population on the GPU and cannot let the
library allocate device memory (a device-side GA loop inside a fixed memory
budget, or a framework whose pooled allocator owns the device).  The test
passes device buffers owned by the caller (torch tensors here) straight
through the C ABI and compares the result with the regular entry point,
sr_eval_mse, on two calls in a row, so that a second call reusing the fixed
scratch after a first one is covered.  The file is collected last and needs
nothing from the other tests.
"""
import ctypes

import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import _lib, synth
from symbolic_regression_gpu_b200 import opcodes as op
from symbolic_regression_gpu_b200.population import Population

pytestmark = pytest.mark.gpu

# Same bound as the plain-vs-batched comparison in test_gpu_parity.py.
REL_TOL = 1e-6


def _device_population(torch, pop: Population):
    """tokens int32, values float32 (constants / variable indices), offsets int64."""
    dev = torch.device("cuda", 0)
    tok = torch.from_numpy(pop.tokens.astype(np.int32)).to(dev)
    val = torch.from_numpy(pop.values.astype(np.float32)).to(dev)
    off = torch.from_numpy(pop.offsets.astype(np.int64)).to(dev)
    return tok, val, off


def _noalloc(torch, pop: Population, X: np.ndarray, offsets=None):
    """One call through the C ABI; offsets (int64, num_exprs + 1) replaces the
    population's own to plant inconsistent ones."""
    dev = torch.device("cuda", 0)
    tok, val, off = _device_population(torch, pop)
    if offsets is not None:
        off = torch.from_numpy(np.asarray(offsets, np.int64)).to(dev)
    Xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).to(dev)
    out = torch.full((pop.num_exprs,), -1.0, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = _lib.lib.sr_eval_mse_device_noalloc(
        ctypes.c_void_p(tok.data_ptr()), ctypes.c_void_p(val.data_ptr()),
        ctypes.c_void_p(off.data_ptr()), pop.num_exprs, ctypes.c_void_p(Xd.data_ptr()),
        X.shape[1], X.shape[0] - 1, X.shape[1], ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(stream.cuda_stream))
    return st, out.cpu().numpy()


def _check_against_regular(mse, ref):
    assert (np.isnan(mse) == np.isnan(ref)).all()
    ok = np.isfinite(ref)
    rel = np.abs(mse[ok].astype(np.float64) - ref[ok]) / np.maximum(np.abs(ref[ok]), 1e-30)
    assert (rel <= REL_TOL).all(), rel.max()


def test_noalloc_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    torch.cuda.init()
    first = synth.plain_workload(seed=61, E=300, N=50_000)
    second = synth.batched_workload(seed=62, E=500, N=30_000, generations=2)
    with sg.Evaluator(device=0) as ev:
        for w in (first, second):
            ev.set_data(w.X)
            ref = ev.eval_mse(w.population)
            st, mse = _noalloc(torch, w.population, w.X)
            assert st == _lib.SR_OK, _lib.status_string(st)
            _check_against_regular(mse, ref)


def test_noalloc_rejects_malformed_and_oversized():
    torch = pytest.importorskip("torch")
    torch.cuda.init()
    w = synth.plain_workload(seed=63, E=8, N=1000)
    bad = Population.from_lists(list(w.population) + [([op.ADD, -1], [0.0, 0.0])])
    st, mse = _noalloc(torch, bad, w.X)
    assert st == _lib.SR_ERR_MALFORMED_EXPRESSION
    assert np.isnan(mse[-1])
    # The population size bound is checked before any device work.
    dev = torch.device("cuda", 0)
    out = torch.empty(1, dtype=torch.float32, device=dev)
    st = _lib.lib.sr_eval_mse_device_noalloc(
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(out.data_ptr()), _lib.SR_NOALLOC_MAX_EXPRS + 1,
        ctypes.c_void_p(out.data_ptr()), 1, 0, 1, ctypes.c_void_p(out.data_ptr()), None)
    assert st == _lib.SR_ERR_UNSUPPORTED
    # A well-formed call right after still works.
    st, mse = _noalloc(torch, w.population, w.X)
    assert st == _lib.SR_OK


def test_noalloc_rejects_inconsistent_offsets_and_checks_without_datapoints():
    torch = pytest.importorskip("torch")
    torch.cuda.init()
    w = synth.plain_workload(seed=64, E=6, N=2000)
    pop = w.population
    good = pop.offsets.copy()
    # Offsets that step backwards or past off[E] are rejected for their
    # expression only; every other expression is still evaluated.
    back = good.copy()
    back[2] = back[3] + 1          # expression 1 runs into 3, expression 2 ends before it starts
    st, mse = _noalloc(torch, pop, w.X, offsets=back)
    assert st == _lib.SR_ERR_MALFORMED_EXPRESSION
    assert np.isnan(mse[1]) and np.isnan(mse[2])
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        ref = ev.eval_mse(pop)
    keep = [0, 3, 4, 5]
    _check_against_regular(mse[keep], ref[keep])
    beyond = good.copy()
    beyond[-2] = beyond[-1] + 5    # the last two expressions would end / start past off[E]
    st, mse = _noalloc(torch, pop, w.X, offsets=beyond)
    assert st == _lib.SR_ERR_MALFORMED_EXPRESSION
    assert np.isnan(mse[-1]) and np.isnan(mse[-2])
    # With no datapoints the structure is still checked: a malformed
    # expression is reported, and every MSE is NaN (no valid datapoint).
    X0 = np.zeros((w.X.shape[0], 0), np.float32)
    bad = Population.from_lists(list(pop) + [([op.SIN], [0.0])])
    st, mse = _noalloc(torch, bad, X0)
    assert st == _lib.SR_ERR_MALFORMED_EXPRESSION
    assert np.isnan(mse).all()
    st, mse = _noalloc(torch, pop, X0)
    assert st == _lib.SR_OK
    assert np.isnan(mse).all()


def test_noalloc_large_population_fewer_datapoint_blocks():
    """5,000 expressions x 40,000 datapoints: the partial sums of 256 datapoint
    blocks would not fit the fixed array, so the call runs fewer blocks (52),
    each covering more datapoints; the results match the regular entry point."""
    torch = pytest.importorskip("torch")
    torch.cuda.init()
    w = synth.batched_workload(seed=65, E=5000, N=40_000, generations=1)
    assert (_lib.SR_NOALLOC_SCRATCH_BYTES - 256) // 16 // 5000 < (40_000 + 127) // 128
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        ref = ev.eval_mse(w.population)
    for _ in range(2):
        st, mse = _noalloc(torch, w.population, w.X)
        assert st == _lib.SR_OK, _lib.status_string(st)
        _check_against_regular(mse, ref)


def test_noalloc_maximum_population():
    """SR_NOALLOC_MAX_EXPRS expressions (one datapoint block each) on a small
    dataset: the largest population the fixed array holds."""
    torch = pytest.importorskip("torch")
    torch.cuda.init()
    base = synth.plain_workload(seed=66, E=48, N=300)
    reps = -(-_lib.SR_NOALLOC_MAX_EXPRS // base.population.num_exprs)
    from symbolic_regression_gpu_b200.population import concat
    pop = concat([base.population] * reps).slice(0, _lib.SR_NOALLOC_MAX_EXPRS)
    with sg.Evaluator(device=0) as ev:
        ev.set_data(base.X)
        ref = ev.eval_mse(base.population)
    st, mse = _noalloc(torch, pop, base.X)
    assert st == _lib.SR_OK, _lib.status_string(st)
    want = np.resize(ref, pop.num_exprs)
    _check_against_regular(mse, want)
