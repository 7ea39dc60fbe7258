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
