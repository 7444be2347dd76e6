"""Per size class choice of the squaring plan, by measurement.

A plan is the split of the length-N transform: ``lr = 0`` keeps a whole test
in one CTA's shared memory (n <= 14); ``lr = 1`` keeps it in the shared
memory of a thread-block cluster (eight CTAs at n = 12, sixteen at n = 13, 14,
2^(n-13) CTAs for 15 <= n <= 17); ``100 +
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

The tuner is native (gfc_batch_tune, genefer22_b200/csrc/gf_host.cu): it
captures K squarings of each candidate plan into a CUDA graph, replays it
between CUDA events and keeps the fastest (device time per squaring, the
minimum over a few replays).  It squares register 0 of the batch in place, so
tune a batch before loading its tests.  This module caches the choice per
(n, test count, tests on the 3-prime set, packed range) in memory and,
optionally, in a JSON file.
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from ._lib import GfcError, check, lib
from .transform import Batch

SMALL_MAX_LOGN = 14


PLAN_CLUSTER = 1
PLAN_SIX = 100
PLAN_PACKED = 200
PLAN_PACKED_SIX = 300


def packed_ok(b: int, n: int) -> bool:
    """Whether base b at size n fits packed digits (two per coefficient), the
    range the engine enforces for plans 200 + lr and 300 + lr2 (gfc_packed_range)."""
    return lib().gfc_packed_range(int(b), int(n)) == 1


def candidates(n: int) -> List[int]:
    """Plans the engine accepts for size n (gfc_plan_candidates), in the order
    the tuner measures them."""
    out = (ctypes.c_int32 * 32)()
    cnt = ctypes.c_size_t(0)
    check(lib().gfc_plan_candidates(int(n), out, 32, ctypes.byref(cnt)))
    return [int(out[i]) for i in range(cnt.value)]


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
        plans = (ctypes.c_int32 * 32)()
        times = (ctypes.c_float * 32)()
        cnt = ctypes.c_size_t(0)
        bestc = ctypes.c_int32(0)
        check(lib().gfc_batch_tune(bt.handle, self.squarings, self.replays, plans, times, 32, ctypes.byref(cnt),
                                   ctypes.byref(bestc)))
        us: Dict[int, float] = {int(plans[i]): float(times[i]) for i in range(min(cnt.value, 32))}
        best = int(bestc.value)
        self.cache[k] = {"lr": best, "us": {str(a): v for a, v in us.items()}}
        self._save()
        return TuneResult(bt.n, bt.count, wide, best, us, packable)
