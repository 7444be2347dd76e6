"""A small, fixed squaring case for kernel profiles: one batch of `count`
tests of size n (bases seeded uniform in [10^6, bmax), even), register 0 of
each test loaded with seeded random balanced digits (so that every carry path
does its full work), then `squarings` squarings with the given plan.

    python -m genefer22_b200.profile_case --n 22 --count 1 --squarings 2
"""
from __future__ import annotations

import argparse

import numpy as np

from ._lib import lib
from .transform import Batch


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, required=True)
    ap.add_argument("--count", type=int, default=1)
    ap.add_argument("--bmax", type=int, default=35_000_000)
    ap.add_argument("--plan", type=int, default=-1, help="-1: the default plan")
    ap.add_argument("--squarings", type=int, default=2)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--read", action="store_true", help="read register 0 back at the end (carry fix-up kernel)")
    ap.add_argument("--mulscalar", type=int, default=0, help="then squareMul by this a (|a| > 2: k_mulscalar)")
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    bases = [int(x) & ~1 for x in rng.integers(1_000_000, a.bmax, size=a.count)]
    with Batch(bases, a.n) as bt:
        if a.plan >= 0:
            bt.set_plan(a.plan)
        for i, b in enumerate(bases):
            bt.put(i, rng.integers(-(b // 2), b // 2, size=1 << a.n, dtype=np.int64).astype(np.int32))
        bt.square(False, a.squarings)
        if a.mulscalar:
            # gfc_square_mul on the batch handle: every test squared, then times a
            rc = lib().gfc_square_mul(bt.handle, a.mulscalar)
            if rc != 0:
                raise RuntimeError(lib().gfc_last_error().decode())
        if a.read:
            bt.get(0, 0)
        bt.sync()
        print(f"n={a.n} tests={a.count} plan={bt.plan()} widths={sorted(set(bt.widths().tolist()))} squarings={a.squarings}")


if __name__ == "__main__":
    main()
