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
