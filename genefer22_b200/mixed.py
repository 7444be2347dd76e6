"""Uneven batches: tests of different sizes n in flight together.

Tests are grouped into size classes (one ``Batch`` per n, its plan chosen by
the ``Autotuner``); every class has its own CUDA stream and replays one graph
per Gerbicz-Li block, and the host enqueues the classes' blocks round-robin,
so the classes' launches overlap on the device.  A test's arithmetic depends
only on its own registers, base and exponent bits, so its residue is the same
alone and in the mix; ``run_alone`` computes it alone for that comparison.

The reference runs one test per process (src/genefer.h:1360-1480); mixing
sizes has no counterpart there.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import gint
from .autotune import Autotuner, TuneResult
from .genefer import BatchPRP, Job, Result
from .transform import Batch


@dataclass
class SizeClass:
    n: int
    index: List[int]                 # positions of the class's tests in the job list
    batch: Batch
    prp: BatchPRP
    tune: Optional[TuneResult] = None
    blocks: List[int] = field(default_factory=list)


@dataclass
class MixedStats:
    seconds: float = 0.0
    digit_squarings: float = 0.0     # sum over tests of N * (exponent bits), padding excluded
    per_class: Dict[int, dict] = field(default_factory=dict)

    @property
    def rate(self) -> float:
        return self.digit_squarings / self.seconds if self.seconds > 0 else 0.0


class MixedBatch:
    """Runs ``jobs`` (any mix of n) with one Batch and graph per size class.

    B: Gerbicz-Li block length, an int for every class, or None for genefer's
    B_GerbiczLi of each class's longest exponent (src/genefer.h:467-471).
    """

    def __init__(self, jobs: Sequence[Job], B: Optional[int] = None, tuner: Optional[Autotuner] = None,
                 device: int = 0, num_regs: int = 3):
        self.jobs = list(jobs)
        self.device = device
        self.classes: List[SizeClass] = []
        by_n: Dict[int, List[int]] = {}
        for i, j in enumerate(self.jobs):
            by_n.setdefault(int(j.n), []).append(i)
        for n in sorted(by_n):
            idx = by_n[n]
            bt = Batch([self.jobs[i].b for i in idx], n, num_regs=num_regs, device=device)
            tr = tuner.tune(bt) if tuner is not None else None
            exps = [(self.jobs[i].words, self.jobs[i].nbits) for i in idx]
            prp = BatchPRP(bt, B, exps=exps)
            self.classes.append(SizeClass(n, idx, bt, prp, tr, prp.schedule()))

    def close(self):
        for c in self.classes:
            c.prp._graph = None
            c.batch.close()
        self.classes = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def plans(self) -> Dict[int, int]:
        return {c.n: c.batch.plan() for c in self.classes}

    def run(self, validate: bool = True) -> List[Result]:
        """Runs every test to the end of its exponent; results in job order."""
        for c in self.classes:
            c.prp.load()
        for c in self.classes:            # record the graphs before timing anything
            if len(c.blocks) > 1:
                c.prp.block_graph()
        t0 = time.perf_counter()
        step = 0
        left = True
        while left:
            left = False
            for c in self.classes:
                if step >= len(c.blocks):
                    continue
                left = True
                cnt = c.blocks[step]
                if step == len(c.blocks) - 1:
                    c.batch.square_exp(cnt)
                elif cnt == c.prp.B:
                    c.prp.block_graph().launch()
                else:
                    c.batch.square_exp(cnt)
                    c.batch.gl_step()
            step += 1
        done = {}
        for c in self.classes:
            c.batch.sync()
            done[c.n] = time.perf_counter() - t0
        self.stats = MixedStats(seconds=max(done.values()) if done else 0.0)
        for c in self.classes:
            ds = float(sum(self.jobs[i].nbits for i in c.index)) * (1 << c.n)
            self.stats.digit_squarings += ds
            self.stats.per_class[c.n] = {"tests": len(c.index), "plan": c.batch.plan(), "B": c.prp.B,
                                         "blocks": len(c.blocks), "digit_squarings": ds, "synced_at_s": done[c.n]}
        out: List[Optional[Result]] = [None] * len(self.jobs)
        for c in self.classes:
            for k, r in zip(c.index, c.prp.results(validate)):
                out[k] = r
        return out                          # type: ignore[return-value]

    def residues(self) -> List[np.ndarray]:
        """Canonical digits of every test's residue (after ``run``), in job order."""
        out: List[Optional[np.ndarray]] = [None] * len(self.jobs)
        for c in self.classes:
            for k, i in enumerate(c.index):
                out[i] = c.prp.canon[k]
        return out                          # type: ignore[return-value]


def run_alone(job: Job, B: int, device: int = 0, plan: Optional[int] = None):
    """The same exponentiation as in a MixedBatch, with the test alone in its
    batch; returns (Result without GL, canonical residue digits)."""
    with Batch([job.b], job.n, num_regs=3, device=device) as bt:
        if plan is not None:
            bt.set_plan(plan)
        prp = BatchPRP(bt, B, exps=[(job.words, job.nbits)])
        prp.load()
        prp.run_prp()
        canon = gint.unbalance(bt.get(0, 0), job.b)
        is_prp, r64, o64 = gint.is_one(canon, job.b)
        prp._graph = None
        return Result(job.b, job.n, is_prp, r64, o64, True), canon


# ------------------------------------------------------------------ the uneven workload

SIZE_MIX = {12: 0.40, 13: 0.20, 14: 0.15, 15: 0.10, 16: 0.08, 17: 0.05, 18: 0.02}


def b_limit(n: int) -> int:
    """Largest b genefer tests on CPU at size n (README.md:22); the GPU limit is 2e9."""
    if n <= 15:
        return 2_000_000_000
    return {16: 1_500_000_000, 17: 1_000_000_000, 18: 1_000_000_000, 19: 70_000_000, 20: 55_000_000,
            21: 45_000_000, 22: 35_000_000, 23: 25_000_000}[n]


def uneven_tests(count: int = 256, seed: int = 1004, mix: Dict[int, float] = SIZE_MIX) -> List[tuple]:
    """(b, n) of the uneven workload: n drawn from ``mix``, b even and
    log-uniform in [1024, 2e9) clipped to b_limit(n)."""
    rng = np.random.default_rng(seed)
    ns = np.array(sorted(mix))
    p = np.array([mix[n] for n in ns], dtype=np.float64)
    p /= p.sum()
    out = []
    for _ in range(count):
        n = int(rng.choice(ns, p=p))
        b = int(np.exp(rng.uniform(np.log(1024.0), np.log(2e9))))
        b = min(b, b_limit(n) - 2)
        b -= b & 1
        out.append((max(b, 1024), n))
    return out
