"""Allocation failure at every point of a call sequence (fault injection on
the host, sr_inject_allocation_failure): the failing call returns
SR_ERR_OUT_OF_MEMORY, the process and the GPU carry on, and the same context
afterwards gives the results of an undisturbed run.  No GPU fault is involved:
the injected failure happens before the allocator is reached, and every call
checks its allocations before it launches anything."""
import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import _lib, synth
from symbolic_regression_gpu_b200.evaluator import detect_subtrees
from symbolic_regression_gpu_b200.evolution import DeviceEvolution, evolve_options

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def work():
    w = synth.cache_workload(seed=13, E=256, N=8192, parents=16, shared=8)
    wg = synth.grad_workload(seed=14, E=64, N=4096)
    return w, wg


def _sequence(ev, w, wg, progress):
    """Every allocating entry point once; `progress` records the steps done."""
    r = {}
    ev.set_data(w.X)
    progress.append("data")
    r["batched"] = ev.eval_mse(w.population)
    r["cached1"] = ev.eval_mse(w.population, cache=True, clear_cache=True)
    progress.append("cached1")
    r["cached2"] = ev.eval_mse(w.population, cache=True)
    r["plain"] = ev.eval_mse(w.population, plain=True)
    ev.prepare(w.population)
    ev.launch()
    r["launch"] = ev.read_mse()
    r["sums"] = ev.read_sums()[0]
    r["pred"] = ev.predictions(w.population.slice(0, 8), 0, 512)
    r["fp64"] = ev.eval_mse_fp64(w.population.slice(0, 16))
    _, groups = detect_subtrees(w.population, evaluator=ev)
    r["detect"] = groups["key"]
    progress.append("w done")
    ev.set_data(wg.X)
    progress.append("grad data")
    r["grad_mse"], r["grad"] = ev.eval_grad(wg.population)
    r["adam"], _ = ev.optimize_constants(wg.population, steps=2)
    de = DeviceEvolution(ev, 64, evolve_options(wg.num_vars, seed=5), stride=64)
    de.init()
    de.evaluate()
    r["evo0"] = de.fitness()
    de.step()
    de.evaluate()
    r["evo1"] = de.fitness()
    return r


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f":
        return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)
    return np.array_equal(a, b)


def _check(r, base):
    for k, v in base.items():
        if k in ("grad", "adam"):  # FP64 atomics: summation order varies
            fin = np.isfinite(v)
            assert np.array_equal(fin, np.isfinite(r[k])), k
            assert np.allclose(r[k][fin], v[fin], rtol=1e-5, atol=1e-7), k
        else:
            assert _same(r[k], v), k


def _evaluator():
    return sg.Evaluator(device=0, dpt=8, warps_per_block=8)


def test_every_allocation_failure_is_reported_and_recoverable(work):
    w, wg = work
    with _evaluator() as ev:
        base = _sequence(ev, w, wg, [])
    failures = 0
    for n in range(1, 400):
        progress = []
        with _evaluator() as ev:
            assert _lib.lib.sr_inject_allocation_failure(n) == _lib.SR_OK
            try:
                _sequence(ev, w, wg, progress)
                completed = True
            except sg.SrError as e:
                assert e.status == _lib.SR_ERR_OUT_OF_MEMORY, (n, progress, str(e))
                completed = False
            finally:
                _lib.lib.sr_inject_allocation_failure(0)
            if completed:
                break
            failures += 1
            if progress and progress[-1] in ("data", "cached1"):
                # A cached evaluation right after the failure: no subtree the
                # failed call registered may be read without being computed.
                assert _same(ev.eval_mse(w.population, cache=True), base["batched"]), n
            _check(_sequence(ev, w, wg, []), base)
    else:
        pytest.fail("the sequence never completed under injection")
    assert failures > 20  # the sequence allocates at many points
