"""Subtree-cache path (reference evaluate_gpu_mse, src/cleaned/cl_gpu_eval.cu:332-564)."""
import numpy as np
import pytest

from oracle import oracle
import symbolic_regression_gpu_b200 as sg
from symbolic_regression_gpu_b200 import synth

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    return ((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))).all()


@pytest.fixture(scope="module")
def work():
    return synth.cache_workload(seed=31, E=1500, N=30_000, parents=80, shared=16)


def test_cached_equals_uncached(work):
    with sg.Evaluator(device=0, dpt=8, warps_per_block=8) as ev:
        ev.set_data(work.X)
        plain = ev.eval_mse(work.population)
        cached = ev.eval_mse(work.population, cache=True, clear_cache=True)
        st = ev.stats
    assert st.num_subtrees > 0 and st.new_subtrees > 0
    assert st.node_evals_executed < st.node_evals
    # Same operators on the same operands: identical predictions, identical
    # summation order -> identical MSE bits.
    assert _bits_equal(plain, cached)


def test_cached_matches_reference_semantics(work):
    with sg.Evaluator(device=0) as ev:
        ev.set_data(work.X)
        cached = ev.eval_mse(work.population, cache=True, clear_cache=True)
    ref = oracle.mse_f32(work.population, work.X)
    assert (np.isnan(cached) == np.isnan(ref)).all()
    ok = np.isfinite(ref)
    r = np.abs(cached[ok] - ref[ok]) / np.maximum(np.abs(ref[ok]), 1e-30)
    assert np.median(r) <= 1e-7


def test_cache_persists_across_generations(work):
    pop = work.population
    half = pop.slice(0, pop.num_exprs // 2)
    with sg.Evaluator(device=0) as ev:
        ev.set_data(work.X)
        ev.eval_mse(pop, cache=True, clear_cache=True)
        used = ev.stats.cache_slots_used
        assert used > 0
        # Same population again: every detected key is already cached.
        again = ev.eval_mse(pop, cache=True)
        assert ev.stats.new_subtrees == 0
        assert ev.stats.cache_slots_used == used
        # A later generation reuses slots of the earlier one.
        sub = ev.eval_mse(half, cache=True)
        assert ev.stats.cache_slots_used >= used
        ref = ev.eval_mse(half)
        assert _bits_equal(sub, ref)
        # clear_cache drops everything.
        ev.eval_mse(half, cache=True, clear_cache=True)
        assert ev.stats.cache_slots_used == ev.stats.new_subtrees
        assert again.shape == (pop.num_exprs,)


def test_cache_capacity_limit(work):
    with sg.Evaluator(device=0, cache_capacity=5) as ev:
        ev.set_data(work.X)
        cached = ev.eval_mse(work.population, cache=True, clear_cache=True)
        assert ev.stats.cache_slots_used == 5
        plain = ev.eval_mse(work.population)
    assert _bits_equal(cached, plain)


def test_cache_invalidated_by_new_data(work):
    with sg.Evaluator(device=0) as ev:
        ev.set_data(work.X)
        ev.eval_mse(work.population, cache=True, clear_cache=True)
        X2 = work.X.copy()
        X2[:-1] *= 0.5
        ev.set_data(X2)
        cached = ev.eval_mse(work.population, cache=True)
        plain = ev.eval_mse(work.population)
    assert _bits_equal(cached, plain)


def test_prepare_without_launch_leaves_no_phantom_cache_entries(work):
    """A cached prepare inserts the new subtrees' keys, whose values exist only
    once its launch runs.  A second prepare before any launch must not find
    those keys (it would read cache rows nothing has written)."""
    with sg.Evaluator(device=0) as ev:
        ev.set_data(work.X)
        want = ev.eval_mse(work.population, cache=True, clear_cache=True)
        ev.prepare(work.population, cache=True, clear_cache=True)  # never launched
        ev.prepare(work.population, cache=True)
        ev.launch()
        got = ev.read_mse()
        st = ev.stats
    assert st.new_subtrees > 0  # the dropped prepare's subtrees are evaluated again
    assert _bits_equal(got, want)
