"""Expression sharding over a process group (symbolic_regression_gpu_b200/sharding.py).

The split and the all-gather are host logic: they run here as two gloo ranks on
the CPU, each evaluating its slice with the oracle (a stand-in for the GPU
evaluator), and the gathered vector must equal the oracle's MSE of the whole
population bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from symbolic_regression_gpu_b200 import sharding, synth
from symbolic_regression_gpu_b200.population import Population


def test_cost_bounds_cover_and_balance():
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 4, 8):
        for E in (0, 1, 5, 100, 1001):
            lens = rng.integers(1, 128, size=E)
            b = sharding.cost_bounds(lens, world)
            assert b[0] == 0 and b[-1] == E and np.all(np.diff(b) >= 0)
            if E == 0:
                continue
            total = int(lens.sum())
            share = total / world
            for r in range(world):
                tok = int(lens[b[r]:b[r + 1]].sum())
                # a slice exceeds its share by less than its last expression
                assert tok <= share + lens.max() + 1


def test_cost_bounds_rejects_bad_world():
    with pytest.raises(ValueError):
        sharding.cost_bounds([1, 2, 3], 0)


def test_shard_slices_concatenate_to_population():
    w = synth.plain_workload(seed=5, E=97, N=64)
    parts = [sharding.shard(w.population, r, 3) for r in range(3)]
    assert parts[0][1] == 0 and parts[-1][2] == 97
    toks = np.concatenate([p[0].tokens for p in parts])
    assert np.array_equal(toks, w.population.tokens)


class _OracleEvaluator:
    """Oracle-backed stand-in for the GPU evaluator of one rank."""

    def __init__(self):
        self.X = None

    def set_data(self, X):
        self.X = np.array(X, dtype=np.float32)

    def eval_mse(self, pop):
        from oracle import oracle
        return oracle.mse_f32(pop, self.X)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, tokens, values, offsets, X, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        pop = Population(tokens, values, offsets)
        sev = sharding.ShardedEvaluator(_OracleEvaluator())
        # dataset only on rank 0: broadcast to the others
        sev.set_data(X if rank == 0 else None)
        mse = sev.eval_mse(pop)
        np.save(os.path.join(out_dir, f"mse{rank}.npy"), mse)
        np.save(os.path.join(out_dir, f"bounds{rank}.npy"), sev.last_bounds)
        # an empty population gathers to an empty vector
        empty = Population(np.zeros(0, np.int32), np.zeros(0), np.zeros(1, np.int64))
        assert sev.eval_mse(empty).size == 0
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharded_eval_matches_oracle(tmp_path):
    from oracle import oracle
    w = synth.plain_workload(seed=11, E=41, N=300)
    pop = w.population
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), pop.tokens, pop.values,
                                         pop.offsets, w.X, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    ref = oracle.mse_f32(pop, w.X)
    for r in range(world):
        got = np.load(tmp_path / f"mse{r}.npy")
        assert got.shape == ref.shape
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        ok = ~np.isnan(ref)
        assert np.array_equal(got[ok], ref[ok])
        b = np.load(tmp_path / f"bounds{r}.npy")
        assert np.array_equal(b, sharding.cost_bounds(pop.lengths(), world))


# ---- datapoint sharding ---------------------------------------------------------

def test_datapoint_bounds_cover_and_align():
    for world in (1, 2, 3, 8):
        for n in (0, 1, 1000, 4096, 1_000_003):
            d = sharding.datapoint_bounds(n, world, align=1024)
            assert d[0] == 0 and d[-1] == n and np.all(np.diff(d) >= 0)
            assert all(int(x) % 1024 == 0 for x in d[1:-1] if 0 < x < n)
    with pytest.raises(ValueError):
        sharding.datapoint_bounds(10, 0)


def test_combine_sums_adds_in_rank_order_and_marks_empty():
    s = np.array([[1.0, 0.0, 2.0], [3.0, 0.0, 0.0]])
    c = np.array([[1.0, 0.0, 2.0], [1.0, 0.0, 0.0]])
    m = sharding.combine_sums(s, c)
    assert m.dtype == np.float32
    assert m[0] == np.float32(2.0) and np.isnan(m[1]) and m[2] == np.float32(1.0)


class _OracleShardEvaluator:
    """Oracle-backed stand-in for one rank's evaluator over its datapoint shard:
    sums of float squared errors in FP64 (the reference's reduction), and FP64
    gradient sums (the FP64 gradient oracle times the valid count)."""

    def __init__(self):
        self.X = None
        self._pop = None

    def set_data(self, X):
        self.X = np.array(X, dtype=np.float32)

    def eval_sums(self, pop):
        from oracle import oracle
        pred = oracle.predict_f32(pop, self.X)
        y = self.X[-1]
        valid = np.isfinite(pred)
        d = (pred - y[None, :]).astype(np.float32)
        with np.errstate(over="ignore", invalid="ignore"):
            sq = np.where(valid, d * d, np.float32(0)).astype(np.float64)
        return sq.sum(axis=1), valid.sum(axis=1).astype(np.float64)

    def eval_grad(self, pop):
        self._pop = pop

    def read_sums(self):
        from oracle import oracle
        mse, cnt = oracle.mse_f64(self._pop, self.X)
        return np.where(cnt > 0, mse * cnt, 0.0), cnt.astype(np.float64)

    def read_grad_sums(self):
        from oracle import oracle
        _, cnt = oracle.mse_f64(self._pop, self.X)
        _, grad = oracle.grad_f64(self._pop, self.X)
        per_const = np.repeat(cnt, self._pop.constant_counts()).astype(np.float64)
        return np.where(per_const > 0, grad * per_const, 0.0)


def _dp_rank_main(rank, world, port, tokens, values, offsets, X, out_dir, scatter):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        pop = Population(tokens, values, offsets)
        ev = _OracleShardEvaluator()
        sev = sharding.DatapointShardedEvaluator(ev, align=128)
        sev.set_data(None if (scatter and rank != 0) else X)
        lo, hi = int(sev.bounds[rank]), int(sev.bounds[rank + 1])
        assert np.array_equal(ev.X, X[:, lo:hi])
        np.save(os.path.join(out_dir, f"dmse{rank}.npy"), sev.eval_mse(pop))
        mse, grad = sev.eval_grad(pop)
        np.save(os.path.join(out_dir, f"dgmse{rank}.npy"), mse)
        np.save(os.path.join(out_dir, f"dgrad{rank}.npy"), grad)
        empty = Population(np.zeros(0, np.int32), np.zeros(0), np.zeros(1, np.int64))
        assert sev.eval_mse(empty).size == 0
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("scatter", [False, True])
def test_two_rank_gloo_datapoint_sharded_eval_matches_oracle(tmp_path, scatter):
    from oracle import oracle
    w = synth.grad_workload(seed=6, E=37, N=1000)
    pop = w.population
    world = 2
    mp.start_processes(_dp_rank_main, args=(world, _free_port(), pop.tokens, pop.values,
                                            pop.offsets, w.X, str(tmp_path), scatter),
                       nprocs=world, join=True, start_method="spawn")
    ref = oracle.mse_f32(pop, w.X)
    mse64, _ = oracle.mse_f64(pop, w.X)
    _, g64 = oracle.grad_f64(pop, w.X)
    for r in range(world):
        got = np.load(tmp_path / f"dmse{r}.npy")
        assert np.array_equal(np.isnan(got), np.isnan(ref))
        ok = ~np.isnan(ref)
        # two partial FP64 sums instead of one sequential sum: at most one
        # float ulp apart after the division
        assert np.all(np.abs(got[ok] - ref[ok]) <= np.spacing(np.abs(ref[ok])))
        gm = np.load(tmp_path / f"dgmse{r}.npy")
        fin = np.isfinite(mse64)
        assert np.allclose(gm[fin], mse64[fin].astype(np.float32), rtol=2e-7, atol=0)
        gr = np.load(tmp_path / f"dgrad{r}.npy")
        fin_g = np.isfinite(g64)
        assert np.allclose(gr[fin_g], g64[fin_g].astype(np.float32), rtol=1e-6, atol=1e-30)
    assert np.array_equal(np.load(tmp_path / "dmse0.npy"), np.load(tmp_path / "dmse1.npy"),
                          equal_nan=True)
