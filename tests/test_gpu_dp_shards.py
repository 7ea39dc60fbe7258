"""Datapoint sharding through the C ABI (sr_read_sums / sr_read_grad_sums):
two contexts on one GPU, each holding half of the columns of X, stand in for
two ranks (the exchange is host arithmetic, covered by the gloo tests in
test_sharding.py).  The combined result must match one context over all
datapoints: MSE within one float ulp (two FP64 partial sums added instead of
one span-ordered sum), gradients within FP64 summation noise."""
import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import sharding, synth

pytestmark = pytest.mark.gpu


def test_read_sums_divides_to_read_mse_exactly():
    w = synth.batched_workload(seed=9, E=300, N=70_001)
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        mse = ev.eval_mse(w.population)
        s, c = ev.read_sums()
    with np.errstate(invalid="ignore", divide="ignore"):
        again = np.where(c > 0, s / np.maximum(c, 1), np.nan).astype(np.float32)
    assert np.array_equal(again, mse, equal_nan=True)
    assert np.all(c <= w.num_dps)


@pytest.mark.parametrize("cache", [False, True])
def test_two_datapoint_shards_combine_to_the_whole(cache):
    w = synth.cache_workload(seed=3, E=512, N=200_000, parents=32) if cache else \
        synth.batched_workload(seed=5, E=600, N=200_000)
    pop = w.population
    d = sharding.datapoint_bounds(w.num_dps, 2)
    sums, cnts = [], []
    for r in range(2):
        with sg.Evaluator(device=0) as ev:
            ev.set_data(np.ascontiguousarray(w.X[:, d[r]:d[r + 1]]))
            ev.eval_mse(pop, cache=cache)
            s, c = ev.read_sums()
            sums.append(s)
            cnts.append(c)
    got = sharding.combine_sums(np.stack(sums), np.stack(cnts))
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        want = ev.eval_mse(pop)
    assert np.array_equal(np.isnan(got), np.isnan(want))
    ok = np.isfinite(want)
    assert np.all(np.abs(got[ok] - want[ok]) <= np.spacing(np.abs(want[ok])))


def test_two_datapoint_shards_combine_gradients():
    w = synth.grad_workload(seed=4, E=256, N=100_000)
    pop = w.population
    d = sharding.datapoint_bounds(w.num_dps, 2)
    s_all, c_all, g_all = [], [], []
    for r in range(2):
        with sg.Evaluator(device=0) as ev:
            ev.set_data(np.ascontiguousarray(w.X[:, d[r]:d[r + 1]]))
            ev.eval_grad(pop)
            s, c = ev.read_sums()
            s_all.append(s)
            c_all.append(c)
            g_all.append(ev.read_grad_sums())
    cnt = c_all[0] + c_all[1]
    per_const = np.repeat(cnt, pop.constant_counts())
    with np.errstate(invalid="ignore", divide="ignore"):
        grad = np.where(per_const > 0, (g_all[0] + g_all[1]) / np.maximum(per_const, 1), np.nan)
    mse = sharding.combine_sums(np.stack(s_all), np.stack(c_all))
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        want_mse, want_grad = ev.eval_grad(pop)
    ok = np.isfinite(want_mse)
    assert np.all(np.abs(mse[ok] - want_mse[ok]) <= np.spacing(np.abs(want_mse[ok])))
    fin = np.isfinite(want_grad) & np.isfinite(grad)
    assert fin.sum() > 0.9 * np.isfinite(want_grad).sum()
    # FP64 sums in another association: equal to float rounding except where
    # a gradient is a near-total cancellation of its per-datapoint terms.
    rel = np.abs(grad[fin] - want_grad[fin]) / np.maximum(np.abs(want_grad[fin]), 1e-30)
    assert np.median(rel) <= 1e-7
    assert np.quantile(rel, 0.99) <= 1e-5
