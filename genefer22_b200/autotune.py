"""Per size class choice of the squaring plan, by measurement.

A plan is the split of the length-N transform: ``lr = 0`` keeps a whole test
in one CTA's shared memory (n <= 14); ``lr = 1`` keeps it in the shared
memory of a thread-block cluster of 2^(n-13) CTAs (15 <= n <= 17); ``100 +
lr2`` splits the column transform into a 16-point register pass and a
2^lr2-point middle pass (six-step); ``200 + lr`` (four-step) and ``300 + lr2`` (six-step)
pack two base-b digits into one coefficient of a half-length transform over
four primes (valid when every base of the batch lies in the exact range; the
engine refuses it otherwise);
``lr >= 3`` runs the four-step form,
2^lr-point column transforms (radix-16 register groups, 2^lr-point tiles in
shared memory or registers) then 2^(n - lr)-point row transforms, the row
pass carrying the pointwise product.  Without packing, the prime set (2 or
3 primes) follows from each base: the narrowest exact set is the fastest.
The RNS width the tuner does choose is packing: four primes on half as many
points instead of two or three on all of them.

The reference has no counterpart: genefer runs one test per transform with a
fixed GPU kernel split chosen from n (src/transformGPU.h:945-1083).

The tuner captures K squarings of each candidate plan into a CUDA graph,
replays it, and keeps the fastest (device time per squaring, taken as the
minimum over a few replays).  It squares register 0 of the batch in place, so
tune a batch before loading its tests.  Results are cached per
(n, test count, tests on the 3-prime set) in memory and, optionally, in a JSON
file.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from ._lib import GfcError
from .transform import Batch

SMALL_MAX_LOGN = 14


PLAN_CLUSTER = 1
PLAN_SIX = 100
PLAN_PACKED = 200
PLAN_PACKED_SIX = 300


# Prime set 2 of the engine (packed digits): the exact range of plans 200 + lr
# and 300 + lr2 (the engine refuses other bases with GFC_ERR_RANGE).
_P2 = (127 * 2**24 + 1, 63 * 2**25 + 1, 249 * 2**23 + 1, 15 * 2**27 + 1)
_M2 = _P2[0] * _P2[1] * _P2[2] * _P2[3]


def packed_ok(b: int, n: int) -> bool:
    """Whether base b at size n fits packed digits (two per coefficient)."""
    b = int(b)
    return (1 << 20) <= b < (1 << 28) and ((b // 2 + 1) * (b + 1)) ** 2 < (_M2 // 2) // (1 << (int(n) - 1))


def candidates(n: int) -> List[int]:
    """Plans the engine accepts for size n (it rejects the others with GFC_ERR_ARG)."""
    out = [0] if n <= SMALL_MAX_LOGN else []
    if 15 <= n <= 17:
        out.append(PLAN_CLUSTER)
    for lr in range(3, 11):
        lc = n - lr
        if 8 <= lc <= 13:
            out.append(lr)
    for lr in (3, 4):                       # packed digits: four primes, transform of N/2
        if 8 <= n - 1 - lr <= 13:
            out.append(PLAN_PACKED + lr)
    for lr2 in range(3, 8):                 # packed digits, six-step on N/2
        lc = n - 1 - 4 - lr2
        if 8 <= lc <= 13 and max(32, 4096 >> lr2) <= (1 << lc):
            out.append(PLAN_PACKED_SIX + lr2)
    for lr2 in range(3, 8):                 # six-step: 2^4 x 2^lr2 column split
        lc = n - 4 - lr2
        if 8 <= lc <= 13 and max(32, 4096 >> lr2) <= (1 << lc):
            out.append(PLAN_SIX + lr2)
    return out


@dataclass
class TuneResult:
    n: int
    count: int
    wide: int                       # tests on the 3-prime set
    lr: int                         # chosen plan
    us: Dict[int, float] = field(default_factory=dict)   # plan -> microseconds per batch squaring

    packable: bool = False

    def key(self) -> str:
        return key(self.n, self.count, self.wide, self.packable)


def key(n: int, count: int, wide: int, packable: bool = False) -> str:
    return f"n{n}_c{count}_w{wide}" + ("_p" if packable else "")


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, squarings: int = 16, replays: int = 3):
        self.cache_path = cache_path
        self.squarings = int(squarings)
        self.replays = int(replays)
        self.cache: Dict[str, dict] = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def _save(self):
        if self.cache_path:
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)

    def measure(self, bt: Batch, lr: int) -> float:
        """Microseconds per batch squaring of plan lr (graph replay, device-bound)."""
        bt.set_plan(lr)
        K = self.squarings
        g = bt.capture(lambda: bt.square(False, K))
        try:
            g.launch()
            bt.sync()
            best = float("inf")
            for _ in range(self.replays):
                t0 = time.perf_counter()
                g.launch()
                bt.sync()
                best = min(best, time.perf_counter() - t0)
        finally:
            g.close()
        return best / K * 1e6

    def tune(self, bt: Batch, force: bool = False) -> TuneResult:
        """Chooses and sets the fastest plan for bt (before its tests are loaded)."""
        packable = all(packed_ok(b, bt.n) for b in bt.bases)
        wide = int(np.count_nonzero(bt.widths() >= 3))
        k = key(bt.n, bt.count, wide, packable)
        if (not force) and (k in self.cache):
            c = self.cache[k]
            try:
                bt.set_plan(int(c["lr"]))
                return TuneResult(bt.n, bt.count, wide, int(c["lr"]), {int(a): v for a, v in c["us"].items()},
                                  packable)
            except GfcError:
                pass                                  # a plan this batch cannot take: measure
        us: Dict[int, float] = {}
        for lr in candidates(bt.n):
            try:
                us[lr] = self.measure(bt, lr)
            except GfcError:
                continue
        if not us:
            raise GfcError(-1, f"no valid plan for n={bt.n}")
        best = min(us, key=lambda lr: (us[lr], lr))
        bt.set_plan(best)
        bt.set(0)
        self.cache[k] = {"lr": best, "us": {str(a): v for a, v in us.items()}}
        self._save()
        return TuneResult(bt.n, bt.count, wide, best, us, packable)
