"""CUDA-graph replay of prepared launches (sr_options.use_graphs): the graph
runs the same kernels on the same buffers, so results are bit-identical to
direct launches; a new prepare or dataset replaces the graph."""
import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def _same(a, b):
    return ((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all()


def test_graph_replay_matches_direct_launch():
    w = synth.batched_workload(seed=13, E=600, N=50_000)
    w2 = synth.plain_workload(seed=14, E=300, N=20_000)
    with sg.Evaluator(device=0) as ref, sg.Evaluator(device=0, use_graphs=True) as ev:
        for e in (ref, ev):
            e.set_data(w.X)
        want = ref.eval_mse(w.population)
        ev.prepare(w.population)
        for _ in range(3):  # first launch captures, the others replay
            ev.launch()
            assert _same(ev.read_mse(), want)
            # the timing events are nodes of the graph
            whole_ms, kern_ms = ev.last_launch_times()
            assert whole_ms > 0 and 0 < kern_ms <= whole_ms
        assert ev.stats.kernel_launches >= 2
        # new population on the same data: recaptured
        want_sub = ref.eval_mse(w.population.slice(0, 200))
        ev.prepare(w.population.slice(0, 200))
        ev.launch()
        ev.launch()
        assert _same(ev.read_mse(), want_sub)
        # new dataset: the old graph (old buffers) must not be replayed
        for e in (ref, ev):
            e.set_data(w2.X)
        want2 = ref.eval_mse(w2.population)
        ev.prepare(w2.population)
        ev.launch()
        ev.launch()
        assert _same(ev.read_mse(), want2)


@pytest.mark.parametrize("mode", [_lib.SR_GRAD_CHECKPOINT, _lib.SR_GRAD_RECOMPUTE])
def test_graph_replay_gradient(mode):
    w = synth.grad_workload(seed=15, E=256, N=30_000)
    with sg.Evaluator(device=0) as ref, sg.Evaluator(device=0, use_graphs=True) as ev:
        for e in (ref, ev):
            e.set_data(w.X)
        m0, g0 = ref.eval_grad(w.population, mode=mode)
        ev.prepare(w.population, gradient=True, grad_mode=mode)
        for _ in range(2):
            ev.launch()
            m1 = ev.read_mse()
            g1 = ev.read_grad()
            assert _same(m1, m0)
            # FP64 atomic adds across spans: their order may differ between
            # runs, which moves the FP32 result by at most an ulp or two
            fin = np.isfinite(g0)
            assert np.array_equal(fin, np.isfinite(g1))
            assert _ulps(g1[fin], g0[fin]).max() <= 2


def test_failed_dataset_replacement_drops_the_prepared_graph():
    """A dataset call that fails after its checks (here: a NULL row in the
    row-pointer form) leaves the context with no dataset and no prepared
    launch, never a captured graph pointing into the old X."""
    import ctypes
    w = synth.batched_workload(seed=12, E=200, N=30_000)
    with sg.Evaluator(device=0, use_graphs=True) as ev:
        ev.set_data(w.X)
        ev.prepare(w.population)
        ev.launch()
        want = ev.read_mse()
        V, N = w.num_vars, w.num_dps
        rows = (ctypes.POINTER(ctypes.c_float) * (V + 1))()
        keep = [np.ascontiguousarray(w.X[v]) for v in range(V + 1)]
        for v in range(V):
            rows[v] = keep[v].ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        rows[V] = ctypes.POINTER(ctypes.c_float)()  # NULL y row
        st = _lib.lib.sr_set_data_rows(ev._ctx, rows, V, N)
        assert st == _lib.SR_ERR_INVALID_ARGUMENT
        assert _lib.lib.sr_launch(ev._ctx) == _lib.SR_ERR_INVALID_ARGUMENT  # nothing prepared
        with pytest.raises(sg.SrError) as ei:
            ev.eval_mse(w.population)
        assert ei.value.status == _lib.SR_ERR_NO_DATA
        ev.set_data(w.X)
        ev.prepare(w.population)
        ev.launch()
        assert _same(ev.read_mse(), want)
