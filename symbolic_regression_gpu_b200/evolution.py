"""The generation loop on the device: evaluate, rank, breed, repeat.

The reference runs its evolution loop on the host (src/cleaned/cl_sr_system.cpp:
150-330) and packs every generation into InputInfo for the evaluator.
``DeviceEvolution`` keeps the population in device memory (slot layout:
expression i has ``lengths[i]`` tokens at ``tokens[i, :]``, float values at
``values[i, :]``) and runs each generation as library calls on the evaluator's
stream: ``sr_prepare_device_population`` (device-side compile) + ``sr_launch``
(the batched interpreter) + ``sr_evolve_step`` (ranking, elites, tournaments,
subtree mutation / crossover).  The host only reads back what it asks for.

PyTorch provides the device buffers; all computation is libsr_eval.so.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional

import numpy as np

from . import _lib
from .evaluator import Evaluator
from .population import Population


def evolve_options(num_vars: int, **overrides) -> _lib.sr_evolve_options:
    """The reference's parameters (sr_evolve_options_init) with overrides;
    ``unary_ops`` / ``binary_ops`` take token lists."""
    o = _lib.sr_evolve_options()
    _lib.check(_lib.lib.sr_evolve_options_init(ctypes.byref(o), num_vars), what="options")
    for k, v in overrides.items():
        if k in ("unary_ops", "binary_ops"):
            arr = getattr(o, k)
            if len(v) > len(arr):
                raise ValueError(f"{k}: at most {len(arr)} operators")
            for i, t in enumerate(v):
                arr[i] = int(t)
            setattr(o, "n_unary" if k == "unary_ops" else "n_binary", len(v))
        else:
            setattr(o, k, v)
    return o


class DeviceEvolution:
    """A population bred and evaluated on the GPU of ``evaluator``.

    ``evaluator.set_data`` must have been called.  ``stride`` defaults to
    ``2 * max_tokens + 2`` (room for the generator's budget-exhausted leaves).
    """

    def __init__(self, evaluator: Evaluator, num_exprs: int, options=None,
                 stride: Optional[int] = None, **overrides):
        import torch

        if evaluator.num_vars is None:
            raise ValueError("evaluator has no dataset: call set_data first")
        self.ev = evaluator
        self.opts = options if options is not None else evolve_options(evaluator.num_vars,
                                                                       **overrides)
        self.E = int(num_exprs)
        self.stride = int(stride) if stride else min(2 * self.opts.max_tokens + 2,
                                                     _lib.SR_EVOLVE_MAX_STRIDE)
        dev = torch.device("cuda", self._device_index())
        self._bufs = [
            (torch.zeros((self.E, self.stride), dtype=torch.int32, device=dev),
             torch.zeros((self.E, self.stride), dtype=torch.float32, device=dev),
             torch.zeros((self.E,), dtype=torch.int32, device=dev))
            for _ in range(2)
        ]
        torch.cuda.synchronize(dev)  # buffers exist before the library stream uses them
        self.cur = 0
        self.generation = 0
        self._evaluated = False

    def _device_index(self) -> int:
        import torch
        return torch.cuda.current_device() if getattr(self.ev, "device", -1) < 0 else self.ev.device

    @staticmethod
    def _ptr(t) -> ctypes.c_void_p:
        return ctypes.c_void_p(t.data_ptr())

    def _check(self, status, what):
        _lib.check(status, self.ev._ctx, what)

    # ---- steps ------------------------------------------------------------
    def init(self):
        """Generation 0: random expressions (reference generate_random_expression)."""
        t, v, n = self._bufs[self.cur]
        self._check(_lib.lib.sr_evolve_init(self.ev._ctx, ctypes.byref(self.opts), self.E,
                                            self.stride, self._ptr(t), self._ptr(v),
                                            self._ptr(n)), "sr_evolve_init")
        self.generation = 0
        self._evaluated = False

    def load(self, pop: Population):
        """Start from a host population (values are used as float32)."""
        import torch
        if pop.num_exprs != self.E:
            raise ValueError("population size differs")
        lens = pop.lengths()
        if lens.max(initial=0) > self.stride:
            raise ValueError("an expression is longer than the stride")
        tok = np.zeros((self.E, self.stride), np.int32)
        val = np.zeros((self.E, self.stride), np.float32)
        for i in range(self.E):
            a, b = int(pop.offsets[i]), int(pop.offsets[i + 1])
            tok[i, :b - a] = pop.tokens[a:b]
            val[i, :b - a] = pop.values[a:b]
        self.ev.synchronize()
        t, v, n = self._bufs[self.cur]
        t.copy_(torch.from_numpy(tok))
        v.copy_(torch.from_numpy(val))
        n.copy_(torch.from_numpy(lens.astype(np.int32)))
        torch.cuda.synchronize(t.device)
        self._evaluated = False

    def evaluate(self):
        """Compile the current population on the device and evaluate it
        (asynchronous after the compile; fitness stays on the device)."""
        t, v, n = self._bufs[self.cur]
        self._check(_lib.lib.sr_prepare_device_population(self.ev._ctx, self._ptr(t), self._ptr(v),
                                                          self._ptr(n), self.E, self.stride),
                    "sr_prepare_device_population")
        self.ev._E = self.E
        self.ev.launch()
        self._evaluated = True

    def step(self):
        """Breed the next generation from the last evaluation's fitness."""
        if not self._evaluated:
            raise RuntimeError("evaluate() the current population first")
        src, dst = self._bufs[self.cur], self._bufs[1 - self.cur]
        fit = ctypes.c_void_p(self.ev.device_mse_ptr())
        self.generation += 1
        self._check(_lib.lib.sr_evolve_step(
            self.ev._ctx, ctypes.byref(self.opts), self.generation, self.E, self.stride, fit,
            self._ptr(src[0]), self._ptr(src[1]), self._ptr(src[2]),
            self._ptr(dst[0]), self._ptr(dst[1]), self._ptr(dst[2])), "sr_evolve_step")
        self.cur = 1 - self.cur
        self._evaluated = False

    def run(self, generations: int, record: bool = True) -> List[Dict[str, float]]:
        """`generations` rounds of evaluate + step, then a final evaluation;
        returns per-generation best / median finite MSE when `record`."""
        hist = []
        for _ in range(generations):
            self.evaluate()
            if record:
                hist.append(self._summary(self.ev.read_mse()))
            self.step()
        self.evaluate()
        if record:
            hist.append(self._summary(self.ev.read_mse()))
        return hist

    @staticmethod
    def _summary(mse: np.ndarray) -> Dict[str, float]:
        fin = mse[np.isfinite(mse)]
        return {"best": float(fin.min()) if fin.size else float("nan"),
                "median": float(np.sort(fin)[fin.size // 2]) if fin.size else float("nan"),
                "finite": int(fin.size)}

    # ---- host views ------------------------------------------------------------
    def population(self) -> Population:
        """The current population, copied to the host (float values widened)."""
        self.ev.synchronize()
        t, v, n = self._bufs[self.cur]
        tok, val, lens = t.cpu().numpy(), v.cpu().numpy(), n.cpu().numpy()
        exprs = [(tok[i, :lens[i]], val[i, :lens[i]].astype(np.float64)) for i in range(self.E)]
        return Population.from_lists(exprs)

    def raw(self):
        """(tokens [E, stride], values [E, stride], lengths [E]) as host arrays."""
        self.ev.synchronize()
        t, v, n = self._bufs[self.cur]
        return t.cpu().numpy(), v.cpu().numpy(), n.cpu().numpy()

    def fitness(self) -> np.ndarray:
        return self.ev.read_mse()
