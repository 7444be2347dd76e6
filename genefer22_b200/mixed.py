"""Uneven batches: tests of different sizes n in flight together.

The native request loop (``gfc_server_*``, genefer22_b200/csrc/gf_server.cpp)
schedules them: every test is submitted at once, each size class gets one
pool with a slot per test (its plan chosen by the native autotuner), and the
dispatcher thread launches every class's Gerbicz-Li block as a CUDA graph on
the class's own stream as soon as its previous block is done, so the
classes' launches overlap on the device.  Finished tests are read back and
checked (genefer's Gerbicz-Li check, src/genefer.h:557-615) by the same loop.
A test's arithmetic depends only on its own slot, base and exponent bits, so
its residue is the same alone and in the mix; ``run_alone`` computes it
alone for that comparison.

The reference runs one test per process (src/genefer.h:1360-1480); mixing
sizes has no counterpart there.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import gint
from .autotune import Autotuner
from .exponent import B_GerbiczLi
from .genefer import BatchPRP, Job, Result
from .serve import Request, Server
from .transform import Batch


@dataclass
class MixedStats:
    seconds: float = 0.0
    digit_squarings: float = 0.0     # sum over tests of N * (exponent bits), padding excluded
    per_class: Dict[int, dict] = field(default_factory=dict)

    @property
    def rate(self) -> float:
        return self.digit_squarings / self.seconds if self.seconds > 0 else 0.0


class MixedBatch:
    """Runs ``jobs`` (any mix of n): one pool per size class, a slot per test.

    B: Gerbicz-Li block length shared by the classes, or None for genefer's
    B_GerbiczLi of the longest exponent (src/genefer.h:467-471); tuner: any
    Autotuner turns the native plan tuning on (None keeps the default plans).
    """

    def __init__(self, jobs: Sequence[Job], B: Optional[int] = None, tuner: Optional[Autotuner] = None,
                 device: int = 0, num_regs: int = 3):
        self.jobs = list(jobs)
        self.device = device
        self.B = int(B) if B else B_GerbiczLi(max(int(j.nbits) for j in self.jobs))
        self.tune = tuner is not None
        self.counts: Dict[int, int] = {}
        for j in self.jobs:
            self.counts[int(j.n)] = self.counts.get(int(j.n), 0) + 1
        self._canon: List[Optional[np.ndarray]] = [None] * len(self.jobs)
        self._plans: Dict[int, int] = {}
        self.stats = MixedStats()

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def plans(self) -> Dict[int, int]:
        """Plan of each size class's pool (after ``run``)."""
        return dict(self._plans)

    def run(self, validate: bool = True, warmup: bool = False) -> List[Result]:
        """Runs every test to the end of its exponent; results in job order.
        With ``warmup`` a first wave of one block per test opens the pools, and
        the statistics cover the second wave only."""
        srv = Server(B=self.B, capacity=lambda n: self.counts.get(n, 1), tune=self.tune, validate=validate,
                     validate_group=4, keep_digits=True, device=self.device, idle_close_s=60.0)
        warm = [Request(len(self.jobs) + i, Job.prefix(j.b, j.n, self.B), 0.0) for i, j in enumerate(self.jobs)] \
            if warmup else []
        comps = srv.run([Request(i, j, 0.0) for i, j in enumerate(self.jobs)], warmup=warm)
        st = srv.stats
        self.stats = MixedStats(seconds=max(c.residue_at for c in comps) - min(c.arrival for c in comps),
                                digit_squarings=float(sum((1 << j.n) * j.nbits for j in self.jobs)))
        out: List[Result] = []
        for i, (j, c) in enumerate(zip(self.jobs, comps)):
            self._canon[i] = c.digits
            self._plans[int(j.n)] = c.plan
            out.append(Result(int(j.b), int(j.n), c.is_prp, c.res64, c.old64, True if c.gl_ok is None else c.gl_ok))
        for n, k in sorted(self.counts.items()):
            sub = [c for c in comps if c.n == n]
            self.stats.per_class[n] = {"tests": k, "plan": self._plans.get(n), "B": self.B,
                                       "digit_squarings": float(sum((1 << n) * c.nbits for c in sub)),
                                       "residue_at_s": max(c.residue_at for c in sub)}
        self.server_stats = st
        return out

    def residues(self) -> List[np.ndarray]:
        """Canonical digits of every test's residue (after ``run``), in job order."""
        return list(self._canon)                # type: ignore[return-value]


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
