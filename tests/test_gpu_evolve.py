"""The device-side generation loop (csrc/sr_evolve.cu) against its restatement
(oracle/evolve.py): generation 0, ranking and breeding must match draw for
draw, bit for bit; a population compiled on the device must evaluate to the
same MSE bits as the same population compiled on the host."""
import ctypes

import numpy as np
import pytest

import symbolic_regression_gpu_b200 as sg
from oracle import evolve as oe
from symbolic_regression_gpu_b200 import _lib, synth
from symbolic_regression_gpu_b200.evolution import DeviceEvolution, evolve_options
from symbolic_regression_gpu_b200.population import Population

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _opts_dict(o):
    return dict(num_vars=o.num_vars, max_tokens=o.max_tokens, max_depth=o.max_depth,
                tournament=o.tournament, const_min=o.const_min, const_max=o.const_max,
                prob_leaf=o.prob_leaf, prob_const_leaf=o.prob_const_leaf,
                prob_unary=o.prob_unary, elite_frac=o.elite_frac,
                mutation_prob=o.mutation_prob, unary_ops=list(o.unary_ops[:o.n_unary]),
                binary_ops=list(o.binary_ops[:o.n_binary]), seed=o.seed)


def _same_population(raw, exprs):
    tok, val, lens = raw
    assert lens.tolist() == [len(t) for t, _ in exprs]
    for i, (t, v) in enumerate(exprs):
        n = len(t)
        assert tok[i, :n].tolist() == [int(x) for x in t], i
        assert np.array_equal(val[i, :n].view(np.uint32), np.asarray(v, np.float32).view(np.uint32)), i


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def data():
    w = synth.plain_workload(seed=21, E=8, N=20_000)
    return w


def test_init_and_steps_match_oracle(data):
    with sg.Evaluator(device=0) as ev:
        ev.set_data(data.X)
        o = evolve_options(3, seed=1234)
        de = DeviceEvolution(ev, 300, o, stride=130)
        de.init()
        od = _opts_dict(o)
        want = oe.evolve_init(od, 300, 130)
        _same_population(de.raw(), want)
        rng = np.random.default_rng(4)
        pop = want
        for gen in range(1, 4):
            fit = rng.uniform(0, 5, 300).astype(np.float32)
            fit[rng.integers(0, 300, 40)] = np.nan        # invalid expressions
            fit[rng.integers(0, 300, 40)] = 1.0           # ties
            fit[:3] = np.inf
            f_dev = torch.from_numpy(fit).cuda()
            src, dst = de._bufs[de.cur], de._bufs[1 - de.cur]
            torch.cuda.synchronize()
            _lib.check(_lib.lib.sr_evolve_step(ev._ctx, ctypes.byref(o), gen, 300, 130, _ptr(f_dev),
                                               _ptr(src[0]), _ptr(src[1]), _ptr(src[2]),
                                               _ptr(dst[0]), _ptr(dst[1]), _ptr(dst[2])))
            de.cur = 1 - de.cur
            pop = oe.evolve_step(od, gen, pop, fit, 130)
            _same_population(de.raw(), pop)


def test_small_stride_and_custom_operators_match_oracle(data):
    # stride = max_tokens: generated subtrees that do not fit fall back to
    # the parent, identically on both sides
    with sg.Evaluator(device=0) as ev:
        ev.set_data(data.X)
        o = evolve_options(3, seed=77, max_tokens=20, max_depth=7, mutation_prob=0.6,
                           unary_ops=[10, 11, 32, 27], binary_ops=[1, 2, 3, 8])
        de = DeviceEvolution(ev, 200, o, stride=20)
        de.init()
        od = _opts_dict(o)
        pop = oe.evolve_init(od, 200, 20)
        _same_population(de.raw(), pop)
        de.evaluate()
        fit = de.fitness()
        de.step()
        _same_population(de.raw(), oe.evolve_step(od, 1, pop, fit, 20))


def test_device_compile_matches_host_compile(data):
    w = synth.batched_workload(seed=8, E=500, N=50_000)
    pop = w.population
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        want = ev.eval_mse(pop)
        de = DeviceEvolution(ev, pop.num_exprs, evolve_options(w.num_vars), stride=
                             int(max(pop.lengths().max(), 64)))
        # values travel as float32 on the device path
        pop32 = Population(pop.tokens, pop.values.astype(np.float32).astype(np.float64),
                           pop.offsets)
        want32 = ev.eval_mse(pop32)
        de.load(pop)
        de.evaluate()
        got = de.fitness()
        st = ev.stats
        # The device-resident evaluation records no upload events; reading its
        # stats must leave no CUDA error behind for the next call's launches.
        mse64 = ev.eval_mse_fp64(pop.subset(np.arange(8)))
    assert np.isfinite(mse64).any()
    same = (got.view(np.uint32) == want32.view(np.uint32)) | (np.isnan(got) & np.isnan(want32))
    assert same.all()
    assert st.node_evals == pop.num_tokens * w.num_dps
    fin = np.isfinite(want)
    assert np.median(np.abs(got[fin] - want[fin]) / np.maximum(np.abs(want[fin]), 1e-30)) < 1e-6


def test_device_population_with_invalid_expression_fails(data):
    with sg.Evaluator(device=0) as ev:
        ev.set_data(data.X)
        de = DeviceEvolution(ev, 4, evolve_options(3), stride=16)
        bad = Population.from_lists([([1, -1, -1], [0, 0, 1]), ([1, -1], [0, 0]),
                                     ([10, 0], [0, 1.5]), ([-1], [2])])
        de.load(bad)
        with pytest.raises(sg.SrError) as ei:
            de.evaluate()
        assert ei.value.status == _lib.SR_ERR_MALFORMED_EXPRESSION


def test_evolution_loop_improves_and_keeps_the_best():
    w = synth.plain_workload(seed=3, E=8, N=30_000)
    with sg.Evaluator(device=0) as ev:
        ev.set_data(w.X)
        de = DeviceEvolution(ev, 2000, seed=99)
        de.init()
        hist = de.run(12)
    best = [h["best"] for h in hist]
    # elites are copied unchanged and re-evaluated to the same bits
    assert all(b2 <= b1 for b1, b2 in zip(best, best[1:]))
    assert best[-1] < best[0]
    assert all(h["finite"] > 0 for h in hist)
