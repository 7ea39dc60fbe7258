"""bench.py --gpus N starts N ranks itself (torchrun, one process per GPU,
rendezvous on 127.0.0.1) when it is not already running under torchrun.  On
the CPU the same launcher runs the bench's multi-rank plumbing with gloo
(--check-launch): every rank builds its own seeded shard, the ranks all-gather
one value per expression (the MSE all-gather of the end-to-end step), and rank
0 reports the world it formed and whether the gathered vector is the
concatenation of the shards."""
import json
import os
import subprocess
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_bench_starts_two_ranks_on_cpu():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", MASTER_ADDR="127.0.0.1")
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        env.pop(k, None)
    cmd = [sys.executable, "bench.py", "--gpus", "2", "--check-launch", "--backend", "gloo",
           "--workload", "plain", "--exprs", "40", "--dps", "64"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2
    assert d["gathered"] == 80 and d["gathered_ok"]
