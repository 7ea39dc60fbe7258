"""Expression sharding of one population over the ranks of a process group.

Expressions are independent given the dataset, so a population splits across
GPUs with no exchange inside the evaluation: every rank keeps the whole
dataset (replicated once, optionally broadcast from rank 0) and evaluates a
contiguous slice of the population whose cost (tokens x datapoints) is about
1/world of the total; one all-gather of the per-expression MSE (4 bytes per
expression) then gives every rank the fitness of the whole population, which
the selection step of the evolution loop needs (reference caller:
src/cleaned/cl_sr_system.cpp:207-249, which consumes every MSE of a
generation).

The reference evaluates on one GPU only (src/cleaned/cl_gpu_eval.cu:332-564);
this module is the multi-GPU partition of the same call.  Slices are
contiguous in population order, so the gathered vector is the concatenation
of the slices and needs no permutation.

Datapoint sharding (DatapointShardedEvaluator) is the partition for datasets
larger than one GPU's memory: rank r keeps only the columns [d[r], d[r+1]) of
X and evaluates the whole population on them; every rank then all-gathers the
per-expression FP64 (sum of valid squared errors, valid count) pairs (16 bytes
per expression per rank) and adds them in rank order, so the result is the
same on every rank and from run to run.  Gradients combine the same way
(FP64 gradient sums over the valid datapoints, divided by the total count).
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

from .population import Population


def cost_bounds(lengths: Sequence[int], world: int) -> np.ndarray:
    """Boundaries b[0]=0 <= b[1] <= ... <= b[world]=E of contiguous slices
    with about equal token counts (the evaluation cost of an expression is
    proportional to its length; every expression sees the same datapoints).

    Slice r is [b[r], b[r+1]).  The boundary of rank r is the first
    expression whose preceding token count reaches r/world of the total, so
    no slice exceeds its share by more than one expression."""
    if world < 1:
        raise ValueError("world must be >= 1")
    lens = np.asarray(lengths, dtype=np.int64)
    E = int(lens.size)
    if np.any(lens < 0):
        raise ValueError("negative expression length")
    before = np.concatenate(([0], np.cumsum(lens)))  # tokens before expression i
    total = int(before[-1])
    b = np.empty(world + 1, dtype=np.int64)
    b[0], b[world] = 0, E
    for r in range(1, world):
        target = (total * r + world - 1) // world  # ceil(total * r / world)
        b[r] = int(np.searchsorted(before, target, side="left"))
    np.maximum.accumulate(b, out=b)
    np.minimum(b, E, out=b)
    return b


def shard(pop: Population, rank: int, world: int) -> Tuple[Population, int, int]:
    """The slice of `pop` that `rank` evaluates: (sub-population, begin, end)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    b = cost_bounds(pop.lengths(), world)
    lo, hi = int(b[rank]), int(b[rank + 1])
    return pop.slice(lo, hi), lo, hi


def gather_mse(local: np.ndarray, bounds: np.ndarray, group=None, device=None) -> np.ndarray:
    """All-gather the per-expression MSE slices (slice r = bounds[r]:bounds[r+1])
    into the full float32 vector on every rank.

    Slices are padded to the largest one for the collective (all_gather needs
    equal sizes) and un-padded here.  `device` is the tensor device the
    backend wants (a CUDA device for NCCL, CPU for gloo)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if bounds.size != world + 1:
        raise ValueError("bounds must have world+1 entries")
    sizes = np.diff(bounds)
    rank = dist.get_rank(group)
    if local.size != sizes[rank]:
        raise ValueError(f"rank {rank}: local MSE has {local.size} entries, slice has {sizes[rank]}")
    width = int(max(int(sizes.max()), 1))
    dev = torch.device("cpu") if device is None else torch.device(device)
    buf = torch.full((width,), float("nan"), dtype=torch.float32, device=dev)
    if local.size:
        buf[: local.size] = torch.from_numpy(np.ascontiguousarray(local, dtype=np.float32)).to(dev)
    out = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    parts = [out[r][: int(sizes[r])].cpu().numpy() for r in range(world)]
    return np.concatenate(parts) if parts else np.empty(0, np.float32)


class ShardedEvaluator:
    """One rank's view of a population evaluation sharded over a process group.

    ``evaluator`` is this rank's :class:`~symbolic_regression_gpu_b200.Evaluator`
    (bound to this rank's GPU) or any object with ``set_data(X)`` and
    ``eval_mse(pop) -> np.ndarray``.  ``eval_mse`` evaluates this rank's
    cost-balanced slice and returns the MSE of the whole population on every
    rank.
    """

    def __init__(self, evaluator, group=None, device=None):
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("torch.distributed is not initialised")
        self.ev = evaluator
        self.group = group
        self.device = device
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.last_bounds: Optional[np.ndarray] = None

    def set_data(self, X: Optional[np.ndarray], src: int = 0):
        """Replicate the dataset: every rank passes its copy, or only rank
        `src` does (others pass None) and it is broadcast first."""
        import torch
        import torch.distributed as dist

        dev = torch.device("cpu") if self.device is None else torch.device(self.device)
        shape = torch.zeros(2, dtype=torch.int64, device=dev)
        have = torch.tensor([0 if X is None else 1], dtype=torch.int64, device=dev)
        dist.all_reduce(have, group=self.group)
        if int(have.item()) == self.world:
            self.ev.set_data(X)
            return
        if self.rank == src:
            if X is None:
                raise ValueError("the broadcast source rank must pass the dataset")
            shape[0], shape[1] = X.shape[0], X.shape[1]
        dist.broadcast(shape, src=src, group=self.group)
        rows, cols = int(shape[0].item()), int(shape[1].item())
        t = (torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(dev)
             if self.rank == src else torch.empty((rows, cols), dtype=torch.float32, device=dev))
        dist.broadcast(t, src=src, group=self.group)
        self.ev.set_data(t.cpu().numpy())

    def local_slice(self, pop: Population) -> Tuple[Population, np.ndarray]:
        b = cost_bounds(pop.lengths(), self.world)
        lo, hi = int(b[self.rank]), int(b[self.rank + 1])
        return pop.slice(lo, hi), b

    def eval_mse(self, pop: Population, **kw) -> np.ndarray:
        sub, b = self.local_slice(pop)
        local = self.ev.eval_mse(sub, **kw) if sub.num_exprs else np.empty(0, np.float32)
        self.last_bounds = b
        return gather_mse(np.asarray(local, dtype=np.float32), b, self.group, self.device)


def split_counts(bounds: np.ndarray) -> List[int]:
    """Expressions per rank of a bounds vector."""
    return [int(x) for x in np.diff(bounds)]


def datapoint_bounds(num_dps: int, world: int, align: int = 1024) -> np.ndarray:
    """Boundaries d[0]=0 <= ... <= d[world]=num_dps of contiguous datapoint
    shards of about equal size, interior boundaries on multiples of `align`
    (a whole number of the evaluator's datapoint spans)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if num_dps < 0:
        raise ValueError("negative datapoint count")
    d = np.empty(world + 1, dtype=np.int64)
    d[0], d[world] = 0, num_dps
    for r in range(1, world):
        cut = (num_dps * r) // world
        d[r] = min(num_dps, ((cut + align // 2) // align) * align)
    np.maximum.accumulate(d, out=d)
    return d


def combine_sums(sums: np.ndarray, counts: np.ndarray) -> np.ndarray:
    """MSE from per-rank sums and counts [world, E], added in rank order (FP64)
    and divided as the single-GPU finalisation does: float32(sum / count), NaN
    where no datapoint of any shard is valid."""
    s = np.zeros(sums.shape[1], np.float64)
    c = np.zeros(sums.shape[1], np.float64)
    for r in range(sums.shape[0]):
        s += sums[r]
        c += counts[r]
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(c > 0, (s / np.maximum(c, 1.0)), np.nan).astype(np.float32)


def _gather_rows(local: np.ndarray, group=None, device=None) -> np.ndarray:
    """All-gather one float64 vector of equal length from every rank -> [world, n]."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = torch.device("cpu") if device is None else torch.device(device)
    buf = torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64)).to(dev)
    out = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    return np.stack([t.cpu().numpy() for t in out]) if world else np.empty((0, local.size))


class DatapointShardedEvaluator:
    """One rank's view of an evaluation whose datapoints are split over a
    process group (each rank holds only its columns of X).

    ``evaluator`` is this rank's Evaluator (or any object with ``set_data(X)``,
    ``eval_sums(pop) -> (sum, count)`` and, for gradients, ``eval_grad(pop)``,
    ``read_sums()`` and ``read_grad_sums()``)."""

    def __init__(self, evaluator, group=None, device=None, align: int = 1024):
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("torch.distributed is not initialised")
        self.ev = evaluator
        self.group = group
        self.device = device
        self.align = align
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.bounds: Optional[np.ndarray] = None

    def set_data(self, X: Optional[np.ndarray], num_dps: Optional[int] = None, src: int = 0):
        """Give this rank its shard.  Either every rank passes the whole X
        (each keeps its columns), or rank `src` passes it and the others pass
        None: the shards are then scattered from `src` (only a shard crosses
        to each rank)."""
        import torch
        import torch.distributed as dist

        dev = torch.device("cpu") if self.device is None else torch.device(self.device)
        have = torch.tensor([0 if X is None else 1], dtype=torch.int64, device=dev)
        dist.all_reduce(have, group=self.group)
        if int(have.item()) == self.world:
            X = np.asarray(X, dtype=np.float32)
            self.bounds = datapoint_bounds(X.shape[1], self.world, self.align)
            lo, hi = int(self.bounds[self.rank]), int(self.bounds[self.rank + 1])
            self.ev.set_data(np.ascontiguousarray(X[:, lo:hi]))
            return
        shape = torch.zeros(2, dtype=torch.int64, device=dev)
        if self.rank == src:
            if X is None:
                raise ValueError("the scatter source rank must pass the dataset")
            shape[0], shape[1] = X.shape[0], X.shape[1]
        dist.broadcast(shape, src=src, group=self.group)
        rows, cols = int(shape[0].item()), int(shape[1].item())
        self.bounds = datapoint_bounds(cols, self.world, self.align)
        width = int(max(int(np.diff(self.bounds).max()), 1))
        recv = torch.empty((rows, width), dtype=torch.float32, device=dev)
        chunks = None
        if self.rank == src:
            Xa = np.asarray(X, dtype=np.float32)
            chunks = []
            for r in range(self.world):
                c = np.zeros((rows, width), np.float32)
                lo, hi = int(self.bounds[r]), int(self.bounds[r + 1])
                c[:, : hi - lo] = Xa[:, lo:hi]
                chunks.append(torch.from_numpy(c).to(dev))
        dist.scatter(recv, chunks, src=src, group=self.group)
        n = int(self.bounds[self.rank + 1] - self.bounds[self.rank])
        self.ev.set_data(np.ascontiguousarray(recv.cpu().numpy()[:, :n]))

    def eval_mse(self, pop: Population) -> np.ndarray:
        """MSE of every expression over all shards' datapoints, on every rank
        (every rank passes the same population)."""
        if pop.num_exprs == 0:
            return np.empty(0, np.float32)
        s, c = self.ev.eval_sums(pop)
        g = _gather_rows(np.concatenate([np.asarray(s, np.float64), np.asarray(c, np.float64)]),
                         self.group, self.device)
        E = pop.num_exprs
        return combine_sums(g[:, :E], g[:, E:])

    def eval_grad(self, pop: Population):
        """(MSE [E], d MSE / d constants [C]) over all shards' datapoints."""
        if pop.num_exprs == 0:
            return np.empty(0, np.float32), np.empty(0, np.float32)
        self.ev.eval_grad(pop)
        s, c = self.ev.read_sums()
        gs = self.ev.read_grad_sums()
        E = pop.num_exprs
        g = _gather_rows(np.concatenate([np.asarray(s, np.float64), np.asarray(c, np.float64),
                                         np.asarray(gs, np.float64)]), self.group, self.device)
        mse = combine_sums(g[:, :E], g[:, E:2 * E])
        cnt = np.zeros(E, np.float64)
        gsum = np.zeros(g.shape[1] - 2 * E, np.float64)
        for r in range(g.shape[0]):
            cnt += g[r, E:2 * E]
            gsum += g[r, 2 * E:]
        per_const = np.repeat(cnt, pop.constant_counts())
        with np.errstate(invalid="ignore", divide="ignore"):
            grad = np.where(per_const > 0, gsum / np.maximum(per_const, 1.0), np.nan)
        return mse, grad.astype(np.float32)
