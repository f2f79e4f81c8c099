"""Fitting a cohort of subjects concurrently on one GPU.

Each subject (its own channel count n_s and length T_s) gets a context on its
own CUDA stream.  Two ways to advance them:

* persistent (single-model fits in the mixed form): one E-step launch per
  cohort iteration over all subjects' sample tiles, dealt evenly to one CTA
  per SM as (subject, tile range) work items, with each subject's inverse and
  M-step on its own stream around it -- one CUDA graph per cohort iteration
  (engine.PersistentCohort, amica_cohort_*);
* streams: one graph replay per subject, all enqueued before any is waited
  for, so the subjects' E-steps and their small M-step kernels overlap.  The
  autotuner puts each subject's fused E-step in its fastest tile shape
  (autotune.best_tile_shape), then times a few cohort iterations with every
  subject on the whole GPU and with the SMs split in proportion to each
  subject's E-step work, keeps the faster, and restores the starting state.
"""
from __future__ import annotations

import time
from typing import Sequence

import numpy as np

from . import autotune
from .engine import Amica, PersistentCohort


class Cohort:
    def __init__(self, data: Sequence[np.ndarray], M: int = 1, m: int = 3, precision: int = 1,
                 device: int = 0, sm_budget: int | None = None, inits=None, tune: bool = True,
                 grids: Sequence[int] | None = None, persistent: bool = False, **cfg):
        """data[s]: T_s x n_s float32 raw samples of subject s.  inits[s], when
        given, is (A0, c0) for amica_init; else the engine's random start."""
        self.engines: list[Amica] = []
        for s, x in enumerate(data):
            T, n = x.shape
            eng = Amica(n, T, M, m, precision=precision, device=device, **cfg)
            eng.load_data(np.ascontiguousarray(x, dtype=np.float32))
            eng.preprocess()
            self.engines.append(eng)
        self._inits = inits
        self.reset()
        self.persistent = None
        if persistent:
            self.persistent = PersistentCohort(self.engines)
            self.grids, self.timings = [0] * len(self.engines), {}
            return
        if sm_budget is None:
            import torch
            sm_budget = torch.cuda.get_device_properties(device).multi_processor_count
        self.timings = {}
        # each subject's fused E-step in its fastest tile shape (the persistent
        # kernel above runs one shape for all subjects)
        self.tile_shapes = [autotune.best_tile_shape(e) if tune else 0 for e in self.engines]
        if grids is not None:
            self.grids = list(grids)
        elif tune:
            self.grids, self.timings = autotune.tune_cohort(self.engines, sm_budget, self.reset)
        else:
            self.grids = [0] * len(self.engines)
        for eng, g in zip(self.engines, self.grids):
            eng.set_grid(g)

    def reset(self) -> None:
        """Every subject back to its initial state (amica_init)."""
        for s, eng in enumerate(self.engines):
            if self._inits is not None:
                eng.init(*self._inits[s])
            else:
                eng.init()

    def run(self, iters: int) -> list:
        """`iters` EM iterations of every subject; returns each subject's records."""
        if self.persistent is not None:
            outs, self.last_ms = self.persistent.run(iters)
            return outs
        for eng in self.engines:
            eng.run_async(iters)
        return [eng.run_wait() for eng in self.engines]

    def timed_run(self, iters: int) -> tuple[list, float]:
        t0 = time.perf_counter()
        outs = self.run(iters)
        return outs, time.perf_counter() - t0

    def close(self) -> None:
        if self.persistent is not None:
            self.persistent.close()
            self.persistent = None
        for eng in self.engines:
            eng.close()
        self.engines = []
