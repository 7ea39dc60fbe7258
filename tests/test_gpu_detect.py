"""Common-subtree detection on the device (csrc/sr_detect_gpu.cu) against the
host detector, itself pinned bit for bit to the reference's
detect_common_subtrees (tests/test_keys_detect.py): the same groups in the
same order (representative, size, verified count, flat key) and the same
statistics; the subtree-cache path gives the same MSE bits with either."""
import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import synth
from symbolic_regression_gpu_b200.evaluator import detect_subtrees
from symbolic_regression_gpu_b200.population import Population

pytestmark = pytest.mark.gpu


def _check_same(pop, ev, min_size=3, min_freq=10):
    hs, hg = detect_subtrees(pop, min_size, min_freq)
    ds, dg = detect_subtrees(pop, min_size, min_freq, evaluator=ev)
    assert hs == ds
    for k in hg:
        assert np.array_equal(hg[k], dg[k]), k
    return hs


@pytest.mark.parametrize("seed", [0, 1])
def test_device_detection_equals_host(seed):
    w = synth.cache_workload(seed=40 + seed, E=3000, N=1000, parents=120, shared=24)
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        st = _check_same(w.population, ev)
        assert st["num_subtrees"] > 20 and st["coverage"] > 0.2
        # other thresholds, and a batched population with fewer repeats
        _check_same(w.population, ev, min_size=5, min_freq=3)
        b = synth.batched_workload(seed=9 + seed, E=2000, N=1000)
        _check_same(b.population, ev)


def test_device_detection_edge_cases():
    with sg.Evaluator(device=0) as ev:
        ev.set_data(np.zeros((3, 64), np.float32))
        # equal hash inputs with different constants, -0.0 / +0.0, single leaves
        exprs = []
        for k in range(30):
            exprs.append(([1, 3, -1, 0, 0], [0, 0, 0, 2.0, -0.0 if k % 2 else 0.0]))
            exprs.append(([0], [1.0]))
        pop = Population.from_lists(exprs)
        st = _check_same(pop, ev)
        assert st["num_subtrees"] >= 2
        _check_same(Population.from_lists([([0], [1.0])]), ev)


def test_cached_eval_with_device_detection_matches_host_detection():
    w = synth.cache_workload(seed=31, E=1500, N=30_000, parents=80, shared=16)
    with sg.Evaluator(device=0) as a, sg.Evaluator(device=0, device_detect=True) as b:
        for e in (a, b):
            e.set_data(w.X)
        ma = a.eval_mse(w.population, cache=True, clear_cache=True)
        mb = b.eval_mse(w.population, cache=True, clear_cache=True)
        assert a.stats.num_subtrees == b.stats.num_subtrees > 0
        assert a.stats.coverage == b.stats.coverage
    same = (ma.view(np.uint32) == mb.view(np.uint32)) | (np.isnan(ma) & np.isnan(mb))
    assert same.all()
