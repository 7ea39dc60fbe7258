"""Device microbenchmarks behind the bench's roofline figures
(sr_measure_pipes, sr_measure_operator_rates): positive, ordered as the
operators' costs are, and the accurate-operator bound of a population below
the measured interpreter time."""
import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import _lib, synth
from symbolic_regression_gpu_b200.evaluator import operator_bound_seconds

pytestmark = pytest.mark.gpu


def test_operator_rates_are_ordered_by_cost():
    with sg.Evaluator(device=0) as ev:
        fp32, sfu, nsm = ev.measure_pipes()
        r = ev.measure_operator_rates([0, 1, 3, 8, 10, 32, 22, 27])
        with pytest.raises(sg.SrError) as ei:
            ev.measure_operator_rates([33])
    assert ei.value.status == _lib.SR_ERR_BAD_TOKEN
    assert nsm > 0 and fp32 > sfu > 0
    assert all(v > 0 for v in r.values())
    # an add costs about the harness's own add; sin / exp / log / division cost more
    assert r[1] > 0.3 * r[0]
    for op in (8, 10, 32, 22):
        assert r[op] < r[1]
    assert r[0] <= 1.2 * fp32  # the harness issues at least one FP32 add per evaluation


def test_operator_bound_is_below_the_interpreter_time():
    w = synth.batched_workload(seed=3, E=2000, N=200_000)
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        ev.prepare(w.population)
        ev.launch()
        ev.read_mse()
        ev.launch()
        ev.read_mse()
        _, kern_ms = ev.last_launch_times()
        fp32, _, _ = ev.measure_pipes()
        ops = sorted({0} | {int(t) for t in np.unique(w.population.tokens) if t > 0})
        rates = ev.measure_operator_rates(ops)
    bound_ms = operator_bound_seconds(w.population, w.num_dps, rates, fp32) * 1e3
    assert 0 < bound_ms < kern_ms
