"""Benchmark: population fitness evaluation, node-evals/s on B200.

One step = one generation's evaluation of the whole batched population (10,000
expressions of 3-63 tokens, 5 variables, 1M datapoints): every expression on
every datapoint, reduced to per-expression MSE, through the persistent
interpreter kernel plus the span-combine kernel.  A node-eval is one token of
an original expression evaluated at one datapoint.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one rank per GPU (when not started by torchrun, bench.py starts
torchrun itself); every rank evaluates its own seeded shard of the population
(weak scaling, no collective on the data path; the end-to-end step ends with
the MSE all-gather).  `--impl reference` times the reference's own CPU
evaluator (evaluate_cpu_mse, compiled unchanged into oracle/_ref) on the host
cores instead.  `--check-launch` runs the multi-rank plumbing alone (any
backend, no GPU needed) and prints the ranks it formed.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-evals/s fwd and fwd+adjoint at <=1e-5 rel err vs FP64 oracle, 1 B200"
UNIT = "node-evals/s"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "plain", "cache", "grad", "large"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU work of the CPU-baseline sample")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the forward+adjoint figures")
    ap.add_argument("--no-cache-figures", action="store_true",
                    help="skip the subtree-cache figures")
    ap.add_argument("--no-evolution", action="store_true",
                    help="skip the device generation-loop figures")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 100,000 x 4M population (forward, fused forward+adjoint, "
                         "plain kernel; about a minute)")
    ap.add_argument("--no-plain-baseline", action="store_true",
                    help="skip the plain per-expression kernel on the headline population")
    ap.add_argument("--no-plain-config", action="store_true",
                    help="skip the plain-forward workload at full size (1,000 x 100k)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's own GPU evaluators on the headline population")
    ap.add_argument("--check-launch", action="store_true",
                    help="form the ranks, build each rank's shard, all-gather a per-expression "
                         "vector, print the ranks (no GPU work; gloo works)")
    ap.add_argument("--backend", default="nccl", help="process-group backend of --check-launch")
    ap.add_argument("--exprs", type=int, default=0,
                    help="population size override (profiling cases)")
    ap.add_argument("--dps", type=int, default=0,
                    help="with --profile-launch: datapoint count override")
    ap.add_argument("--cached", action="store_true",
                    help="with --profile-launch: evaluate through the subtree cache")
    ap.add_argument("--dpt", type=int, default=0, help="force datapoints per thread")
    ap.add_argument("--warps", type=int, default=0, help="force evaluating warps per block")
    ap.add_argument("--profile-launch", action="store_true",
                    help="prepare and run a single evaluation, no timing (for ncu)")
    ap.add_argument("--grad-mode", choices=["none", "checkpoint", "recompute",
                                            "reverse_checkpoint", "reverse_recompute"],
                    default="none",
                    help="with --profile-launch: run the fused forward + adjoint instead")
    return ap.parse_args()


_T0 = time.perf_counter()


def _progress(what: str):
    """One progress line on stderr (stdout carries only the JSON result)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {what}", file=sys.stderr, flush=True)


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")),
            int(os.environ.get("WORLD_SIZE", "1")))


def make_workload(name: str, rank: int, exprs: int = 0, dps: int = 0):
    from symbolic_regression_gpu_b200 import synth
    fn = synth.WORKLOADS[name]
    seeds = {"plain": 1, "batched": 2, "cache": 3, "grad": 4, "large": 5}
    kw = {"E": exprs} if exprs > 0 else {}
    if dps > 0:
        kw["N"] = dps
    return fn(seed=seeds[name] + 1000 * rank, **kw)


def relaunch_under_torchrun(args) -> int:
    """--gpus N > 1 without a torchrun environment: start N ranks of this same
    command under torchrun (one process per GPU, rendezvous on 127.0.0.1) and
    return its exit status.  Rank 0 prints the JSON line."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1",
           f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def check_launch(args) -> int:
    """The multi-rank plumbing of the bench without GPU work: every rank
    builds its own seeded shard (as the measured run does), the ranks
    all-gather one float per expression (the MSE all-gather of the end-to-end
    step, here the expressions' token counts) and rank 0 checks the gathered
    vector against the shards it rebuilds itself and prints the ranks."""
    import datetime

    import torch
    import torch.distributed as dist

    from symbolic_regression_gpu_b200 import sharding
    rank, local_rank, world = dist_env()
    dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=60))
    dev = torch.device("cuda", local_rank) if args.backend == "nccl" else torch.device("cpu")
    w = make_workload(args.workload, rank, args.exprs, args.dps)
    local = np.diff(w.population.offsets).astype(np.float32)
    E = w.population.num_exprs
    bounds = np.arange(world + 1, dtype=np.int64) * E
    got = sharding.gather_mse(local, bounds, device=dev)
    if rank == 0:
        want = np.concatenate([np.diff(make_workload(args.workload, r, args.exprs,
                                                     args.dps).population.offsets)
                               for r in range(world)]).astype(np.float32)
        print(json.dumps({"n_gpus": world, "backend": args.backend, "exprs_per_rank": E,
                          "gathered": int(got.size),
                          "gathered_ok": bool(np.array_equal(got, want))}))
    dist.barrier()
    dist.destroy_process_group()
    return 0


def profile_launch(args):
    """One prepared evaluation on GPU 0, nothing timed (the ncu capture case)."""
    from symbolic_regression_gpu_b200 import Evaluator, _lib
    w = make_workload(args.workload, 0, args.exprs, args.dps)
    with Evaluator(device=0, dpt=args.dpt, warps_per_block=args.warps) as ev:
        ev.set_data(w.X)
        if args.grad_mode == "none":
            ev.prepare(w.population, cache=args.cached, clear_cache=args.cached)
        else:
            mode = (_lib.SR_GRAD_CHECKPOINT if args.grad_mode.endswith("checkpoint")
                    else _lib.SR_GRAD_RECOMPUTE)
            if args.grad_mode.startswith("reverse"):
                mode |= _lib.SR_GRAD_REVERSE_ONLY
            ev.prepare(w.population, gradient=True, grad_mode=mode)
        ev.launch()
        mse = ev.read_mse()
        st = ev.stats
        print(json.dumps({"workload": w.name, "grad_mode": args.grad_mode,
                          "exprs": w.population.num_exprs,
                          "num_dps": w.num_dps, "dpt": st.dpt,
                          "warps_per_block": st.warps_per_block, "blocks": st.blocks,
                          "work_items": st.work_items, "kernel_ms": st.eval_kernel_time_ms,
                          "finite_mse": int(np.isfinite(mse).sum())}))
    return 0


def config_of(w, world: int, flush: str):
    return {"workload": w.name, "exprs_per_gpu": w.population.num_exprs,
            "global_exprs": w.population.num_exprs * world,
            "tokens_per_gpu": int(w.population.num_tokens),
            "mean_len": round(float(w.meta["len_mean"]), 2), "num_vars": w.num_vars,
            "num_dps": w.num_dps, "x_range": w.meta.get("x_range"),
            "ops": "+ - * loose_div sin cos exp_clamp80 loose_log loose_sqrt",
            "parallelism": f"expr-shard x{world}" if world > 1 else "single",
            "l2": flush}


# ---- clocks -------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid=None):
        self.proc = None
        self.out = os.path.join("/tmp", f"sr_clocks_{os.getpid()}.csv")
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "200"]
        if device_uuid:
            cmd += ["-i", device_uuid]
        try:
            self.fh = open(self.out, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.out) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.out)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "samples": len(sm), "reasons": sorted(reasons)}


# ---- CPU baseline ---------------------------------------------------------------

def _reference_population(pop):
    """The reference evaluator has no exp-clamp opcode: map it to its EXP
    (same expf call) for timing."""
    from symbolic_regression_gpu_b200.population import Population
    tok = pop.tokens.copy()
    tok[tok == 32] = 16
    return Population(tok, pop.values, pop.offsets)


def _ulp_distance(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Distance in representable floats between FP32 arrays (0 for two NaNs,
    a large value when exactly one is NaN)."""
    def ordered(x):
        i = np.asarray(x, np.float32).view(np.int32).astype(np.int64)
        return np.where(i < 0, -(i & 0x7FFFFFFF), i)
    d = np.abs(ordered(a) - ordered(b))
    na, nb = np.isnan(a), np.isnan(b)
    return np.where(na & nb, 0, np.where(na | nb, 1 << 40, d))


def _import_generators_only():
    """Make the package's pure-Python workload generators (synth, population,
    opcodes) importable without running the package __init__, which loads
    libsr_eval.so: the reference arm must not map the product library."""
    import types
    if "symbolic_regression_gpu_b200" in sys.modules:
        return
    pkg = types.ModuleType("symbolic_regression_gpu_b200")
    pkg.__path__ = [os.path.join(ROOT, "symbolic_regression_gpu_b200")]
    sys.modules["symbolic_regression_gpu_b200"] = pkg


def _rule_summary(r: dict) -> dict:
    n = max(int(r.get("expressions", r.get("datapoints", 0))), 1)
    out = dict(r)
    out["exempt_flagged_frac"] = r["exempt_flagged"] / n
    out["exempt_conditioning_frac"] = r["exempt_conditioning"] / n
    return out


def parity_figures(ev, w, sample, ours_mse, ref_mse, threads, patched):
    """Parity of the GPU path against the reference on the CPU-baseline sample
    (outside the timed region), under the condition-aware rule (oracle
    error_bound / mse_parity / datapoint_parity):
      * MSE against the reference's evaluate_cpu_mse on the whole sample (raw
        agreement), and the rule on its first 96 expressions over all
        datapoints;
      * per datapoint against the reference's evaluate_single_expr on 512
        expressions x 4,096 datapoints;
      * the reduction error alone (our MSE against an FP64 sum of our own FP32
        predictions);
      * accuracy against the FP64 evaluation under the rule's mode 1 on the
        same 96 expressions."""
    from oracle import oracle
    out = {"reference": ("evaluate_cpu_mse / evaluate_single_expr with the one added "
                         "exp-clamp case (oracle/_ref/libref_expc.so)") if patched else
           "the oracle's restatement of evaluate_cpu_mse (pinned bit for bit by the goldens)"}
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(np.asarray(ours_mse, np.float64) - ref_mse) / np.maximum(np.abs(ref_mse), 1e-300)
    both = np.isfinite(ours_mse) & np.isfinite(ref_mse)
    out["mse_vs_reference_cpu"] = {
        "expressions": int(sample.num_exprs), "finite": int(both.sum()),
        "median_rel": float(np.median(r[both])) if both.any() else None,
        "frac_le_1e-6": float(np.mean(r[both] <= 1e-6)) if both.any() else None,
        "nan_pattern_equal": bool(np.array_equal(np.isnan(ours_mse), np.isnan(ref_mse))),
        "inf_pattern_equal": bool(np.array_equal(np.isinf(ours_mse), np.isinf(ref_mse)))}
    k = min(96, sample.num_exprs)
    sub = sample.slice(0, k)
    b = oracle.error_bound(sub, w.X, mode=0, threads=threads)
    out["mse_rule"] = _rule_summary(oracle.mse_parity(ours_mse[:k], ref_mse[:k],
                                                      b["mse_bound"], b["flagged"]))
    out["mse_rule"]["datapoints"] = int(w.num_dps)
    ns = min(4096, w.num_dps)
    sub2 = sample.slice(0, min(512, sample.num_exprs))
    Xs = np.ascontiguousarray(w.X[:, :ns])
    ours = ev.predictions(sub2, 0, ns)
    theirs = oracle.refx_predict(sub2, Xs, threads) if patched else oracle.predict_f32(sub2, Xs)
    bb = oracle.error_bound(sub2, Xs, mode=0, per_datapoint=True, threads=threads)
    rd = oracle.datapoint_parity(ours, theirs, bb["bound"], bb["flag"])
    u = _ulp_distance(ours, theirs)
    rd = _rule_summary(rd)
    rd.update({"expressions": int(sub2.num_exprs), "datapoints_per_expression": int(ns),
               "bit_identical_frac": float(np.mean(u == 0)),
               "frac_le_4ulp": float(np.mean(u <= 4)),
               "raw_gt_4ulp": int(np.count_nonzero(u > 4))})
    out["per_datapoint"] = rd
    red = sample.slice(0, min(16, sample.num_exprs))
    pred = ev.predictions(red)
    sums = oracle.mse_of_predictions(pred, w.X[w.num_vars])
    del pred
    ours_red = np.asarray(ours_mse[:red.num_exprs], np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        rr = np.abs(ours_red - sums) / np.maximum(np.abs(sums), 1e-300)
    rr = rr[np.isfinite(rr)]
    out["reduction_error"] = {"expressions": int(red.num_exprs),
                              "max_rel": float(rr.max()) if rr.size else None}
    m64 = ev.eval_mse_fp64(sub)
    b1 = oracle.error_bound(sub, w.X, mode=1, threads=threads)
    out["accuracy_rule_vs_fp64"] = _rule_summary(
        oracle.mse_parity(ours_mse[:k], m64, b1["mse_bound"], b1["flagged"],
                          bar=oracle.FP64_BAR))
    return out


def cpu_baseline(w, target_s: float, threads: int):
    """The reference CPU evaluator (oracle/_ref, compiled -O3) on a seeded
    expression subset over the full datapoint range: its evaluate_cpu_mse
    with the one added exp-clamp case when that build exists (so that the
    same run's MSEs serve as the parity reference), else the unchanged build
    with the exp-clamp opcode timed as its EXP (same expf call)."""
    from oracle import oracle
    patched = oracle.reference_expc_available()
    pop = w.population if patched else _reference_population(w.population)
    fn = oracle.refx_mse if patched else oracle.ref_mse
    E = pop.num_exprs
    rng = np.random.default_rng(7)
    order = rng.permutation(E)
    # Probe the rate, then size the sample to ~target_s of CPU work.
    n_probe = max(threads, min(E, 16))
    probe = pop.subset(order[:n_probe])
    t0 = time.perf_counter()
    fn(probe, w.X, threads=threads)
    rate = probe.num_tokens * w.num_dps / max(time.perf_counter() - t0, 1e-6)
    tokens_target = rate * target_s / w.num_dps
    mean_len = pop.num_tokens / E
    n = int(max(threads, min(E, tokens_target / mean_len)))
    sample = pop.subset(order[:n])
    t0 = time.perf_counter()
    ref = fn(sample, w.X, threads=threads)
    dt = time.perf_counter() - t0
    value = sample.num_tokens * w.num_dps / dt
    ref_mse = np.asarray(ref[0], np.float32)
    what = ("reference evaluate_cpu_mse (src/cleaned/cl_cpu_eval.cpp) with the one added "
            "exp-clamp case" if patched else
            "reference evaluate_cpu_mse (src/cleaned/cl_cpu_eval.cpp) unchanged, exp_clamp80 "
            "timed as the reference EXP opcode")
    return {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
            "_sample_index": order[:n], "_sample_mse": ref_mse, "_patched": patched,
            "sample": f"{n} of {E} expressions (seeded subset) x all {w.num_dps} datapoints, "
                      f"{dt:.1f} s; {what}, compiled -O3, THREADS={threads}"}


def plain_config_figures(ev, torch, flush_buf, sr_stream, threads):
    """The plain-forward workload at full size (1,000 ramped half-and-half
    expressions, 3 variables, 100,000 datapoints): forward and plain-kernel
    node-evals/s, and every MSE against the reference's under the rule (the
    reference evaluator with the exp-clamp case, all 1,000 x 100,000, about a
    second on the host cores)."""
    from oracle import oracle
    w = make_workload("plain", 0)
    pop = w.population
    node_evals = pop.num_tokens * w.num_dps
    ev.set_data(w.X)
    res = {"workload": "plain", "exprs": pop.num_exprs, "num_dps": w.num_dps,
           "num_vars": w.num_vars}
    for name, kw in (("fwd", {}), ("plain_kernel", {"plain": True})):
        ev.prepare(pop, **kw)
        _timed_launches(ev, torch, flush_buf, sr_stream, 2)
        ms = statistics.mean(_timed_launches(ev, torch, flush_buf, sr_stream, 5))
        res[name] = {"value": node_evals / (ms * 1e-3), "unit": UNIT, "ms": ms}
    res["fwd"]["vs_plain_kernel"] = res["plain_kernel"]["ms"] / res["fwd"]["ms"]
    ev.prepare(pop)
    ev.launch()
    mse = ev.read_mse()
    patched = oracle.reference_expc_available()
    t0 = time.perf_counter()
    ref = (oracle.refx_mse(pop, w.X, threads)[0] if patched else
           oracle.mse_f32(pop, w.X, threads))
    cpu_s = time.perf_counter() - t0
    b = oracle.error_bound(pop, w.X, mode=0, threads=threads)
    r = _rule_summary(oracle.mse_parity(mse, ref, b["mse_bound"], b["flagged"]))
    with np.errstate(invalid="ignore", divide="ignore"):
        rel = np.abs(mse.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-300)
    fin = np.isfinite(rel)
    r.update({"reference": "evaluate_cpu_mse with the exp-clamp case" if patched else
              "restatement", "reference_cpu_s": cpu_s, "reference_cpu_threads": threads,
              "median_rel": float(np.median(rel[fin])) if fin.any() else None,
              "frac_le_1e-6": float(np.mean(rel[fin] <= 1e-6)) if fin.any() else None})
    res["parity_full"] = r
    return res


def reference_gpu_figures(w, steps: int = 2):
    """The reference's own GPU evaluators (plain and subtree-cache paths,
    compiled unchanged for sm_100a) on the same population and dataset, in
    their own process (oracle/ref_gpu.py: the reference prints to stdout and
    exits on CUDA errors), chunked within their int32 index limits."""
    import tempfile
    from oracle import ref_gpu
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/libref_gpu.so was not built"}
    why = ref_gpu.check_limits(w.population.tokens.copy(), w.population.values,
                               w.population.offsets, w.num_vars, w.num_dps)
    if why:
        return {"unavailable": why}
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "pop.npz"), os.path.join(td, "res.json")
        np.savez(inp, tokens=w.population.tokens, values=w.population.values,
                 offsets=w.population.offsets, X=w.X)
        t0 = time.perf_counter()
        rc = subprocess.call([sys.executable, "-m", "oracle.ref_gpu", inp, out,
                              "--steps", str(steps)], cwd=ROOT, timeout=900,
                             stdout=subprocess.DEVNULL)
        wall = time.perf_counter() - t0
        if rc != 0 or not os.path.exists(out):
            return {"unavailable": f"the reference GPU process exited with status {rc}"}
        res = json.load(open(out))
    res["process_wall_s"] = wall
    res["what"] = ("evaluate_gpu_simple_wrapper and evaluate_gpu_mse_wrapper (src/cleaned/"
                   "cl_gpu_simple.cu, cl_gpu_eval.cu) compiled unchanged for sm_100a, "
                   "expression chunks with E_chunk x N < 2^31, exp_clamp80 run as EXP; "
                   "kernel_* from the reference's own CUDA events, call_* its wall clock")
    return res


# ---- reference arm ------------------------------------------------------------------

def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    _import_generators_only()
    from oracle import oracle
    if not oracle.reference_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libref_oracle.so was not built"}))
        return 0
    w = make_workload(args.workload, 0, args.exprs)
    threads = os.cpu_count() or 1
    pop = _reference_population(w.population)
    E = pop.num_exprs
    rng = np.random.default_rng(7)
    order = rng.permutation(E)
    # Size one step's sample so warmup+steps stay within a few minutes.
    probe = pop.subset(order[:max(threads, 16)])
    t0 = time.perf_counter()
    oracle.ref_mse(probe, w.X, threads=threads)
    rate = probe.num_tokens * w.num_dps / max(time.perf_counter() - t0, 1e-6)
    per_step_s = min(20.0, 150.0 / max(args.steps + args.warmup, 1))
    n = int(max(threads, min(E, rate * per_step_s / w.num_dps / (pop.num_tokens / E))))
    sample = pop.subset(order[:n])
    for _ in range(args.warmup):
        oracle.ref_mse(sample, w.X, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.ref_mse(sample, w.X, threads=threads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = sample.num_tokens * w.num_dps * len(times) / total
    desc = (f"{n} of {E} expressions (seeded subset) x all {w.num_dps} datapoints per step; "
            f"reference evaluate_cpu_mse compiled -O3, THREADS={threads}; exp_clamp80 timed "
            f"as the reference EXP opcode")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; stands in for AI-Feynman)",
            "config": config_of(w, 1, "n/a (CPU)"), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                             "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---- our arm ----------------------------------------------------------------------

def _timed_launches(ev, torch, flush_buf, sr_stream, steps):
    """Device time (ms) of `steps` launches of the prepared work, L2 flushed
    before each; CUDA events on the evaluator's stream."""
    out = []
    for _ in range(steps):
        with torch.cuda.stream(sr_stream):
            flush_buf.fill_(1.0)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(sr_stream)
        ev.launch()
        e.record(sr_stream)
        e.synchronize()
        out.append(s.elapsed_time(e))
    return out


def adjoint_figures(ev, rank, world, dev, flush_buf, sr_stream, args):
    """node-evals/s of the forward pass and of the gradient launches on the
    constant-optimisation workload, their cost ratio, and 20 Adam steps.
    "checkpoint" / "recompute" are the library's gradient calls in those modes
    (forward mode for expressions with at most 8 constants, which is all of
    this workload); "reverse_checkpoint" / "reverse_recompute" force reverse
    mode (SR_GRAD_REVERSE_ONLY) for every expression."""
    import torch
    from symbolic_regression_gpu_b200 import _lib
    w = make_workload("grad", rank)
    pop = w.population
    node_evals = pop.num_tokens * w.num_dps
    steps = max(3, min(args.steps, 10))
    ev.set_data(w.X)
    ev.prepare(pop)
    _timed_launches(ev, torch, flush_buf, sr_stream, 2)
    fwd_ms = _timed_launches(ev, torch, flush_buf, sr_stream, steps)
    res = {"workload": "grad", "exprs": pop.num_exprs, "num_dps": w.num_dps,
           "num_vars": w.num_vars, "constants": int(np.count_nonzero(pop.tokens == 0)),
           "fwd": {"value": node_evals / (statistics.mean(fwd_ms) * 1e-3), "unit": UNIT,
                   "ms": statistics.mean(fwd_ms)}}
    res["forward_mode_exprs"] = int((pop.constant_counts() <= 8).sum())
    rev = _lib.SR_GRAD_REVERSE_ONLY
    for name, mode in (("checkpoint", _lib.SR_GRAD_CHECKPOINT),
                       ("recompute", _lib.SR_GRAD_RECOMPUTE),
                       ("reverse_checkpoint", _lib.SR_GRAD_CHECKPOINT | rev),
                       ("reverse_recompute", _lib.SR_GRAD_RECOMPUTE | rev)):
        try:
            ev.prepare(pop, gradient=True, grad_mode=mode)
        except _lib.SrError as ex:
            res[name] = {"unavailable": str(ex)}
            continue
        _timed_launches(ev, torch, flush_buf, sr_stream, 2)
        ms = _timed_launches(ev, torch, flush_buf, sr_stream, steps)
        ev.read_mse()  # refreshes ev.stats (launch count of the gradient call)
        grad = ev.read_grad()
        res[name] = {"value": node_evals / (statistics.mean(ms) * 1e-3), "unit": UNIT,
                     "ms": statistics.mean(ms),
                     "cost_vs_fwd": statistics.mean(ms) / statistics.mean(fwd_ms),
                     "launches_per_step": int(ev.stats.kernel_launches),
                     "finite_grad": int(np.isfinite(grad).sum()), "grad_entries": int(grad.size)}
    mse0 = ev.eval_mse(pop)
    t0 = time.perf_counter()
    consts, mse = ev.optimize_constants(pop, steps=20, lr=0.05)
    res["adam20"] = {"wall_ms": (time.perf_counter() - t0) * 1e3,
                     "device_ms": float(ev.stats.gpu_kernel_time_ms),
                     "median_mse_ratio": float(np.nanmedian(mse / mse0)),
                     "improved_frac": float(np.mean(mse[np.isfinite(mse0)] <=
                                                    mse0[np.isfinite(mse0)]))}
    return res


def cache_figures(ev, rank, flush_buf, sr_stream, args):
    """Subtree-cache workload (4,096 expressions derived from 256 parents, 9
    variables, 1M datapoints): one generation with the cross-generation cache
    cleared (detect, fill the new subtrees, evaluate the skeletons) against
    the same population without the cache."""
    import torch
    w = make_workload("cache", rank)
    pop = w.population
    node_evals = pop.num_tokens * w.num_dps
    steps = max(3, min(args.steps, 5))
    ev.set_data(w.X)
    ev.prepare(pop)
    _timed_launches(ev, torch, flush_buf, sr_stream, 1)
    plain_ms = statistics.mean(_timed_launches(ev, torch, flush_buf, sr_stream, steps))
    ev.prepare(pop, cache=True, clear_cache=True)
    _timed_launches(ev, torch, flush_buf, sr_stream, 1)
    cache_ms = statistics.mean(_timed_launches(ev, torch, flush_buf, sr_stream, steps))
    ev.read_mse()
    st = ev.stats
    executed = int(st.node_evals_executed)
    # common-subtree detection alone: host detector vs the device one
    from symbolic_regression_gpu_b200.evaluator import detect_subtrees
    detect_subtrees(pop, evaluator=ev)  # warm-up (buffers, cub)
    t0 = time.perf_counter()
    detect_subtrees(pop)
    t_host = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    detect_subtrees(pop, evaluator=ev)
    t_dev = (time.perf_counter() - t0) * 1e3
    return {"workload": "cache", "exprs": pop.num_exprs, "num_dps": w.num_dps,
            "num_vars": w.num_vars, "no_cache": {"value": node_evals / (plain_ms * 1e-3),
                                                 "unit": UNIT, "ms": plain_ms},
            "cached": {"value": node_evals / (cache_ms * 1e-3), "unit": UNIT, "ms": cache_ms,
                       "executed_node_evals_per_s": executed / (cache_ms * 1e-3)},
            "speedup": plain_ms / cache_ms, "num_subtrees": int(st.num_subtrees),
            "new_subtrees": int(st.new_subtrees), "coverage": float(st.coverage),
            "node_evals": int(node_evals), "node_evals_executed": executed,
            "node_evals_saved": int(node_evals) - executed,
            "detect_ms": {"host": t_host, "device": t_dev,
                          "host_threads": os.cpu_count() or 1}}


def evolution_figures(ev, w, torch, sr_stream, generations=5):
    """The generation loop on the device on the batched dataset: a random
    population of the same size, then per generation the device compile +
    interpreter evaluation and the breeding step, device-timed."""
    import ctypes

    from symbolic_regression_gpu_b200 import _lib
    from symbolic_regression_gpu_b200.evolution import DeviceEvolution
    E = w.population.num_exprs
    ev.set_data(w.X)
    de = DeviceEvolution(ev, E, seed=2024)
    de.init()
    t_prep, t_eval, t_step, best = [], [], [], []
    for g in range(generations + 1):
        t0 = time.perf_counter()
        t, v, n = de._bufs[de.cur]
        ev._check(_lib.lib.sr_prepare_device_population(ev._ctx, ctypes.c_void_p(t.data_ptr()),
                                                         ctypes.c_void_p(v.data_ptr()),
                                                         ctypes.c_void_p(n.data_ptr()), E,
                                                         de.stride),
                   "sr_prepare_device_population")
        t_prep.append((time.perf_counter() - t0) * 1e3)
        ev._E = E
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(sr_stream)
        ev.launch()
        s1.record(sr_stream)
        de._evaluated = True
        mse = ev.read_mse()
        t_eval.append(s0.elapsed_time(s1))
        fin = mse[np.isfinite(mse)]
        best.append(float(fin.min()) if fin.size else float("nan"))
        if g == generations:
            break
        s2 = torch.cuda.Event(enable_timing=True)
        s1.record(sr_stream)
        de.step()
        s2.record(sr_stream)
        s2.synchronize()
        t_step.append(s1.elapsed_time(s2))
    ev.synchronize()
    return {"exprs": E, "num_dps": w.num_dps, "generations": generations,
            "prepare_ms_mean": statistics.mean(t_prep[1:]),
            "eval_ms_mean": statistics.mean(t_eval[1:]),
            "breed_ms_mean": statistics.mean(t_step[1:]) if len(t_step) > 1 else t_step[0],
            "best_mse": best}


def large_figures(device, flush_buf, rank):
    """The large population (100,000 expressions of 3-127 tokens, 0-8
    constants, 10 variables, 4M datapoints): forward, fused forward+adjoint
    and the plain per-expression kernel.  Its own evaluator, with the
    untuned default launch shape (timing candidate shapes on launches of
    seconds would take minutes)."""
    import torch
    from symbolic_regression_gpu_b200 import Evaluator, _lib
    w = make_workload("large", rank)
    pop = w.population
    node_evals = pop.num_tokens * w.num_dps
    ev = Evaluator(device=device)
    sr_stream = torch.cuda.ExternalStream(ev.stream_handle, device=torch.device("cuda", device))
    ev.set_data(w.X)
    res = {"workload": "large", "exprs": pop.num_exprs, "num_dps": w.num_dps,
           "num_vars": w.num_vars, "tokens": int(pop.num_tokens)}
    # The forward pass after one warm-up launch; the fused forward+adjoint and
    # the plain kernel (seconds each) one launch after their prepare.
    for name, kw, n in (("fwd", {}, 2),
                        ("fwd_adjoint", {"gradient": True,
                                         "grad_mode": _lib.SR_GRAD_CHECKPOINT}, 1),
                        ("plain_kernel", {"plain": True}, 1)):
        ev.prepare(pop, **kw)
        ms = _timed_launches(ev, torch, flush_buf, sr_stream, n)[-1]
        res[name] = {"value": node_evals / (ms * 1e-3), "unit": UNIT, "ms": ms}
    res["fwd_adjoint"]["cost_vs_fwd"] = res["fwd_adjoint"]["ms"] / res["fwd"]["ms"]
    res["fwd"]["vs_plain_kernel"] = res["plain_kernel"]["ms"] / res["fwd"]["ms"]
    ev.close()
    return res


def run_ours(args):
    import torch
    rank, local_rank, world = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    from symbolic_regression_gpu_b200 import Evaluator, sharding
    from symbolic_regression_gpu_b200.evaluator import operator_bound_seconds

    w = make_workload(args.workload, rank, args.exprs)
    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    tune_path = os.path.join("/tmp", f"sr_tune_{os.getuid()}.json")
    ev = Evaluator(device=local_rank, autotune=True, tune_cache_path=tune_path, dpt=args.dpt,
                   warps_per_block=args.warps, use_graphs=True)
    sr_stream = torch.cuda.ExternalStream(ev.stream_handle, device=dev)
    ev.set_data(w.X)
    ev.prepare(w.population)  # compile + upload + shape tuning (outside timing)
    _progress("headline population prepared")
    node_evals = w.population.num_tokens * w.num_dps

    def step():
        with torch.cuda.stream(sr_stream):
            flush_buf.fill_(1.0)  # evict the dataset from L2 between steps
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(sr_stream)
        ev.launch()
        e.record(sr_stream)
        e.synchronize()
        launch_ms, kern_ms = ev.last_launch_times()
        return s.elapsed_time(e), kern_ms

    for _ in range(max(args.warmup, 3)):
        step()
    mse = ev.read_mse()
    st = ev.stats
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        uuid = None
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(uuid)
    step_ms, kern_ms = [], []
    for _ in range(args.steps):
        a, b = step()
        step_ms.append(a)
        kern_ms.append(b)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    _progress("headline steps timed")
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = node_evals * world * len(step_ms) / (total_ms * 1e-3)
    mean_kern_ms = sum(kern_ms) / len(kern_ms)

    # Roofline of the interpreter kernel: declared FP32/SFU work per launch
    # against the measured pipe peaks of this device.
    fp32_peak, sfu_peak, nsm = ev.measure_pipes()
    t_fp32 = st.declared_fp32_ops / fp32_peak
    t_sfu = st.declared_sfu_ops / sfu_peak
    bound = "sfu" if t_sfu >= t_fp32 else "fp32"
    ops = st.declared_sfu_ops if bound == "sfu" else st.declared_fp32_ops
    peak = sfu_peak if bound == "sfu" else fp32_peak
    achieved = ops / (mean_kern_ms * 1e-3)
    # Second yardstick: the accurate-operator bound (each operator's CUDA
    # implementation timed alone on this device, no dispatch around it).
    op_list = sorted({0} | {int(t) for t in np.unique(w.population.tokens) if t > 0})
    op_rates = ev.measure_operator_rates(op_list)
    t_ops = operator_bound_seconds(w.population, w.num_dps, op_rates, fp32_peak)
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"interp_{args.workload}_traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except (OSError, ValueError):
            traffic = None

    # Accuracy of the timed results: every expression's MSE against its FP64
    # reference, evaluated on the device (outside the timed region).
    accuracy = None
    if rank == 0:
        rel = ev.accuracy(w.population, mse)
        fin = rel[np.isfinite(rel)]
        accuracy = {"reference": "FP64 evaluation on the device (sr_eval_mse_fp64)",
                    "expressions": int(w.population.num_exprs), "finite": int(fin.size),
                    "median_rel_err": float(np.median(fin)) if fin.size else None,
                    "p99_rel_err": float(np.quantile(fin, 0.99)) if fin.size else None,
                    "frac_le_1e-5": float(np.mean(fin <= 1e-5)) if fin.size else None,
                    "frac_le_1e-6": float(np.mean(fin <= 1e-6)) if fin.size else None}
        ev.prepare(w.population)

    # Plain per-expression kernel on the same population (baseline ratio).
    plain = None
    if not args.no_plain_baseline and rank == 0:
        ev.prepare(w.population, plain=True)
        ev.launch()
        ev.read_mse()
        pm = []
        for _ in range(2):
            a, _ = step()
            pm.append(a)
        plain = {"value": node_evals / (statistics.mean(pm) * 1e-3), "unit": UNIT,
                 "ms_per_step": statistics.mean(pm),
                 "fwd_vs_plain_kernel": statistics.mean(pm) / (total_ms / len(step_ms))}
        ev.prepare(w.population)

    # Forward + adjoint on the constant-optimisation workload (4,096
    # expressions with 1-8 constants, 4 variables, 262,144 datapoints).
    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_figures(ev, rank, world, dev, flush_buf, sr_stream, args)
        _progress("forward+adjoint figures")

    cache = None
    if not args.no_cache_figures:
        cache = cache_figures(ev, rank, flush_buf, sr_stream, args)
        _progress("subtree-cache figures")
    evolution = None
    if not args.no_evolution:
        evolution = evolution_figures(ev, w, torch, sr_stream)
        _progress("device evolution figures")
    large = None
    if not args.no_large:
        large = large_figures(local_rank, flush_buf, rank)
        _progress("large population figures")
        ev.set_data(w.X)
    plain_config = None
    if not args.no_plain_config and rank == 0 and world == 1:
        plain_config = plain_config_figures(ev, torch, flush_buf, sr_stream,
                                            os.cpu_count() or 1)
        _progress("plain workload figures")
        ev.set_data(w.X)

    # End to end through the public API: pinned host dataset and host
    # population in, MSE vector out, every step.
    Xp = torch.empty(w.X.shape, dtype=torch.float32, pin_memory=True)
    Xp.numpy()[...] = w.X
    # With N ranks the population is the concatenation of the ranks' slices;
    # every rank ends the step holding the MSE of all of it (one all-gather,
    # as the selection step of the evolution loop needs).
    bounds = np.arange(world + 1, dtype=np.int64) * w.population.num_exprs
    e2e_times, h2d, d2h = [], 0, 0
    for k in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev.set_data(Xp.numpy())
        out = ev.eval_mse(w.population)
        if world > 1:
            out = sharding.gather_mse(out, bounds, device=dev)
        dt = time.perf_counter() - t0
        if k > 0:
            e2e_times.append(dt)
        h2d = int(Xp.numel() * 4 + ev.stats.h2d_bytes)
        d2h = int(ev.stats.d2h_bytes)
    e2e_s = sum(e2e_times) / len(e2e_times)
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = node_evals * world / e2e_s
    _progress("end-to-end steps")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(w, args.cpu_seconds, os.cpu_count() or 1)
        except (ImportError, FileNotFoundError, OSError) as ex:
            cpu = {"value": None, "unavailable": str(ex)}
        if cpu.get("_sample_index") is not None:
            # The reference's FP32 results on the sample against the same FP64
            # reference, beside ours on the same expressions.
            idx = cpu.pop("_sample_index")
            ref_mse = cpu.pop("_sample_mse")
            sample = w.population.subset(idx)
            ev.set_data(w.X)
            mse64 = ev.eval_mse_fp64(sample)

            def _stats(m):
                with np.errstate(invalid="ignore", divide="ignore"):
                    r = np.abs(np.asarray(m, np.float64) - mse64) / np.maximum(np.abs(mse64), 1e-300)
                r = r[np.isfinite(r)]
                return {"median_rel_err": float(np.median(r)) if r.size else None,
                        "frac_le_1e-5": float(np.mean(r <= 1e-5)) if r.size else None,
                        "finite": int(r.size)}
            cpu["accuracy_vs_fp64"] = {"reference_cpu": _stats(ref_mse),
                                       "this_gpu_same_expressions": _stats(mse[idx])}
            _progress("CPU baseline")
            cpu["parity"] = parity_figures(ev, w, sample, mse[idx], ref_mse,
                                           os.cpu_count() or 1, cpu.pop("_patched"))
            _progress("parity figures")

    reference_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ev.synchronize()
        try:
            reference_gpu = reference_gpu_figures(w)
            _progress("reference GPU figures")
        except (ImportError, OSError, subprocess.SubprocessError) as ex:
            reference_gpu = {"unavailable": str(ex)}
        if "kernel_node_evals_per_s" in reference_gpu.get("simple", {}):
            reference_gpu["ours_fwd_vs_simple_kernel"] = (
                value / reference_gpu["simple"]["kernel_node_evals_per_s"])
        if "kernel_node_evals_per_s" in reference_gpu.get("subtree", {}):
            reference_gpu["ours_fwd_vs_subtree_kernels"] = (
                value / reference_gpu["subtree"]["kernel_node_evals_per_s"])

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": len(step_ms), "warmup": max(args.warmup, 3),
            "ms_per_step": total_ms / len(step_ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; stands in for AI-Feynman)",
            "config": config_of(w, world, "flushed between steps (256 MiB write)"),
            "mode": "fwd",
            "kernel": {"dpt": st.dpt, "warps_per_block": st.warps_per_block,
                       "blocks": st.blocks, "work_items": st.work_items,
                       "interp_ms_mean": mean_kern_ms},
            "roofline": {"bound": bound, "achieved": achieved, "peak": peak, "unit": "op/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "measured on this GPU by sr_measure_pipes "
                                        f"({'MUFU rsqrt' if bound == 'sfu' else 'FP32 FMA'} "
                                        f"microbenchmark, {nsm} SMs)",
                         "model": "declared per-operator FP32/SFU counts (T_min = "
                                  "max(F/P_fp32, S/P_sfu))",
                         "fp32_frac": (st.declared_fp32_ops / (mean_kern_ms * 1e-3)) / fp32_peak,
                         "sfu_frac": (st.declared_sfu_ops / (mean_kern_ms * 1e-3)) / sfu_peak,
                         "accurate_operator_bound": {
                             "ms": t_ops * 1e3, "frac": t_ops * 1e3 / mean_kern_ms,
                             "evals_per_s": {str(k): v for k, v in op_rates.items()},
                             "model": "sum over operator tokens x datapoints of 1/rate of the "
                                      "operator's FP32 semantics timed alone on this GPU "
                                      "(sr_measure_operator_rates), less the harness"}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3},
            "gpu_launches": int(st.kernel_launches) * len(step_ms),
            "clocks": clk,
            "plain_kernel": plain,
            "fwd_adjoint": adjoint,
            "subtree_cache": cache,
            "device_evolution": evolution,
            "large": large,
            "plain_config": plain_config,
            "reference_gpu": reference_gpu,
            "mse_finite": int(np.isfinite(mse).sum()),
            "accuracy_vs_fp64": accuracy,
        }
        print(json.dumps(line))
    ev.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_under_torchrun(args)
    if args.check_launch:
        return check_launch(args)
    if args.profile_launch:
        return profile_launch(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
