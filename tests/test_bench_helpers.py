"""Host-side arithmetic behind the bench's figures (no GPU): the ulp distance
used for per-datapoint parity and the accurate-operator bound."""
import numpy as np

import bench
from symbolic_regression_gpu_b200.evaluator import operator_bound_seconds
from symbolic_regression_gpu_b200.population import Population


def test_ulp_distance():
    one = np.float32(1.0)
    a = np.array([one, -0.0, 0.0, np.nan, np.nan, -one, 1e-45], np.float32)
    b = np.array([np.nextafter(one, np.float32(2)), 0.0, 0.0, np.nan, one,
                  np.nextafter(-one, np.float32(0)), -1e-45], np.float32)
    d = bench._ulp_distance(a, b)
    assert list(d[:4]) == [1, 0, 0, 0]
    assert d[4] >= 1 << 40          # exactly one NaN
    assert d[5] == 1 and d[6] == 2  # across zero: +min -> +0 -> -min


def test_operator_bound_counts_operator_tokens_only():
    # x0 + sin(c): one add and one sin per datapoint; leaves cost nothing
    pop = Population.from_lists([([1, -1, 10, 0], [0, 0, 0, 1.5])])
    rates = {0: 1e13, 1: 5e12, 10: 1e12}
    fp32 = 4e13
    t = operator_bound_seconds(pop, 1000, rates, fp32)
    want = 1000 * ((1 / 5e12 - 1 / 1e13) + (1 / 1e12 - 1 / 1e13))
    assert np.isclose(t, want, rtol=1e-12)
    # an operator no dearer than the harness costs one FP32 instruction
    t2 = operator_bound_seconds(pop, 1000, {0: 1e13, 1: 2e13, 10: 1e12}, fp32)
    assert np.isclose(t2, 1000 * (1 / fp32 + (1 / 1e12 - 1 / 1e13)), rtol=1e-12)
