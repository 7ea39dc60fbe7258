"""Synthetic workloads: seeded, in range (small sizes; full sizes in the bench)."""
import numpy as np

import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import opcodes as op
from symbolic_regression_gpu_b200 import synth


def test_plain_workload_is_seeded_and_shaped():
    a = synth.plain_workload(seed=9, E=60, N=500)
    b = synth.plain_workload(seed=9, E=60, N=500)
    assert (a.population.tokens == b.population.tokens).all()
    assert (a.X == b.X).all()
    assert a.X.shape == (4, 500) and a.X.dtype == np.float32
    assert a.X[:3].min() >= 1.0 and a.X[:3].max() <= 5.0
    used = set(np.unique(a.population.tokens[a.population.tokens > 0]).tolist())
    assert used <= set(op.WORKLOAD_BINARY) | set(op.WORKLOAD_UNARY)
    sg.validate(a.population, 3)


def test_batched_lengths_in_range():
    w = synth.batched_workload(seed=3, E=400, N=100, generations=5)
    L = w.population.lengths()
    assert L.min() >= 3 and L.max() <= 63
    assert 8 <= L.mean() <= 30
    assert synth.repeat_stats(w.population)["repeated_fraction"] > 0.05


def test_grad_workload_constant_counts():
    w = synth.grad_workload(seed=4, E=200, N=128)
    co = w.population.constant_offsets()
    counts = np.diff(co)
    assert counts.min() >= 1 and counts.max() <= 8
    L = w.population.lengths()
    assert L.min() >= 5 and L.max() <= 63


def test_large_workload_shape_small():
    w = synth.large_workload(seed=5, E=300, N=64)
    L = w.population.lengths()
    assert L.min() >= 3 and L.max() <= 127
    counts = np.diff(w.population.constant_offsets())
    assert counts.max() <= 8
    assert w.X.shape == (11, 64)


def test_cache_workload_has_common_subtrees():
    w = synth.cache_workload(seed=3, E=500, N=64, parents=40, shared=10)
    stats, groups = sg.detect_subtrees(w.population, 3, 10)
    assert stats["num_subtrees"] > 5
