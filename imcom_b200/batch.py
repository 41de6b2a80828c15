"""Batched patches: many independent output patches solved side by side on one GPU.

The reference solves one patch (one input stack, one output grid) per program
run (imcom.f90:90-169).  A survey is processed as many such patches, and a
patch of a few thousand input pixels leaves a B200 mostly idle: its
eigensolver is a chain of dependent, latency-bound steps (one grid barrier
pair per Householder column).  Here K worker threads each own a context
(own CUDA stream, own buffers) whose persistent and cooperative kernels are
sized for a share of the SMs (IMCOM_OPT_SM_SHARE), so K patches advance at
once and their kernels fill the GPU together.  Patches are dealt from a
queue, largest n first.

`autotune` measures the patch throughput of candidate configurations --
concurrency x the thread-block cluster that finishes each tridiagonalisation
(IMCOM_OPT_TAIL_CTAS: 16 CTAs hold the longest tail but need 16 free SMs of
one GPC, which contexts working side by side can make wait) -- on a sample of
the batch and returns the fastest (cached per GPU and size class).

Results per patch are those of `Solver.solve` (K, U/S maps, H, the
evaluation counts); only the m-length maps are copied to the host.
"""
from __future__ import annotations

import queue
import threading
import time
from dataclasses import dataclass, field

from . import _lib
from .api import OPT_SM_SHARE, OPT_TAIL_CTAS, Solver

_TUNED: dict = {}


@dataclass
class BatchResult:
    results: list = field(default_factory=list)  # per patch (input order)
    seconds: float = 0.0
    concurrency: int = 1
    sm_share: int = 0
    pixels: int = 0
    timeline: list = field(default_factory=list)  # (patch, worker, t_start, t_end) seconds

    @property
    def patches_per_s(self) -> float:
        return len(self.results) / self.seconds if self.seconds > 0 else 0.0

    @property
    def pixels_per_s(self) -> float:
        return self.pixels / self.seconds if self.seconds > 0 else 0.0


def device_sms(device: int = 0) -> int:
    import torch
    return torch.cuda.get_device_properties(device).multi_processor_count


class BatchSolver:
    """A pool of `concurrency` contexts on one GPU, each with a share of the
    SMs; the contexts (plans, buffers) persist across `solve` calls."""

    def __init__(self, concurrency: int = 4, device: int = 0, setup=None, tail_ctas: int = 0):
        _lib.load()
        self.k = max(1, int(concurrency))
        self.device = device
        self.tail_ctas = int(tail_ctas)
        sms = device_sms(device)
        self.share = sms // self.k if self.k > 1 else 0
        self.solvers = []
        for _ in range(self.k):
            s = Solver(device)
            if self.share:
                s.set_option(OPT_SM_SHARE, self.share)
            if self.tail_ctas:
                s.set_option(OPT_TAIL_CTAS, self.tail_ctas)
            if setup is not None:
                setup(s)
            self.solvers.append(s)

    def _work(self, w, s, jobs, out, errors, solve_kw, t0, timeline):
        try:
            while True:
                try:
                    idx, prob = jobs.get_nowait()
                except queue.Empty:
                    break
                ta = time.perf_counter() - t0
                out[idx] = s.solve(prob, keep=(), **solve_kw)
                out[idx].stage_ms = s.stage_times()
                timeline.append((idx, w, ta, time.perf_counter() - t0))
            s.synchronize()
        except Exception as e:  # reported by the caller
            errors.append(e)

    def solve(self, problems, **solve_kw) -> BatchResult:
        """Solve every problem (largest n first); `solve_kw` goes to
        `Solver.solve` (UnotS, US_max, US_tol, maxnits, learned, ...)."""
        jobs: queue.Queue = queue.Queue()
        for i in sorted(range(len(problems)), key=lambda i: -problems[i].n):
            jobs.put((i, problems[i]))
        out = [None] * len(problems)
        errors: list = []
        timeline: list = []
        k = min(self.k, len(problems))
        t0 = time.perf_counter()
        threads = [threading.Thread(target=self._work,
                                    args=(q, self.solvers[q], jobs, out, errors, solve_kw, t0,
                                          timeline))
                   for q in range(k)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        dt = time.perf_counter() - t0
        if errors:
            raise errors[0]
        return BatchResult(results=out, seconds=dt, concurrency=k, sm_share=self.share,
                           pixels=sum(p.m for p in problems), timeline=sorted(timeline, key=lambda x: x[2]))

    def close(self):
        for s in self.solvers:
            s.close()
        self.solvers = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def solve_patches(problems, concurrency: int = 4, device: int = 0, setup=None,
                  tail_ctas: int = 0, **solve_kw) -> BatchResult:
    """Solve every problem of `problems` (imcom_b200.problem.Problem) with
    `concurrency` contexts side by side (a one-off pool)."""
    with BatchSolver(min(max(1, concurrency), len(problems)), device, setup, tail_ctas) as b:
        return b.solve(problems, **solve_kw)


def size_class(problems) -> int:
    """Bucket of the largest n (powers of two) used as the autotuner cache key."""
    n = max(p.n for p in problems)
    c = 256
    while c < n:
        c *= 2
    return c


@dataclass
class Tuning:
    concurrency: int
    tail_ctas: int                               # IMCOM_OPT_TAIL_CTAS value
    rates: dict = field(default_factory=dict)    # patches/s by (concurrency, tail_ctas)


def autotune(problems, candidates=(1, 2, 4, 6, 8), tails=(0, 8, -1), device: int = 0,
             setup=None, reps: int = 2, **solve_kw) -> Tuning:
    """The configuration (concurrency, tail cluster) with the highest patch
    throughput on `problems` (a sample of the batch).  Each candidate pool is
    warmed up on the sample once (plans, buffers, lazy module loading) and
    then timed on it `reps` times, keeping the best (a GPU shared with other
    work can stall a single pass); the result is cached per (GPU, size
    class)."""
    import torch
    key = (torch.cuda.get_device_name(device), size_class(problems))
    if key in _TUNED:
        return _TUNED[key]
    best, best_rate, rates = None, -1.0, {}
    for k in candidates:
        if k > len(problems):
            break
        for t in tails:
            with BatchSolver(k, device, setup, t) as b:
                b.solve(problems, **solve_kw)
                rate = max(b.solve(problems, **solve_kw).patches_per_s
                           for _ in range(max(1, reps)))
            rates[(k, t)] = rate
            if rate > best_rate:
                best, best_rate = (k, t), rate
    _TUNED[key] = Tuning(best[0], best[1], rates)
    return _TUNED[key]


def make_batch(npatch: int, seed0: int = 0, mask_frac: float = 0.02):
    """The batched-patch workload: `npatch` patches of 4 exposures of side
    16..24 px (seeded), `mask_frac` of the input pixels masked, Gaussian PSF
    sigma ~ U[0.5, 0.8] px per exposure, 24 x 24 outputs at 0.5 px."""
    import numpy as np

    from . import synth
    rng = np.random.default_rng(seed0)
    sides = rng.integers(16, 25, npatch)
    return [synth.make_patch(seed=seed0 + i, side=int(sides[i]), mask_frac=mask_frac)
            for i in range(npatch)]


__all__ = ["BatchSolver", "solve_patches", "autotune", "make_batch", "BatchResult",
           "Tuning", "size_class"]
