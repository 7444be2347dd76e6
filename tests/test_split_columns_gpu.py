"""Kernels in both forms: one thread per column or group for all planes
(batches that fill the GPU) and a thread per (plane, column) or (plane,
group) (single tests and small batches) -- the register column kernels and
the single-CTA kernel.  The engine picks the form from the launch's size, so
the same tests squared one at a time and as one batch run different kernels;
their digits must agree, and one test of each group is checked against the
oracle (restated transformCPUi32), through the carry fix-up path (several
squarings), dup squarings and products."""
import numpy as np
import pytest

from genefer22_b200 import Batch, gint

pytestmark = pytest.mark.gpu


def canon(d, b):
    return gint.unbalance(d, b)


def run(bases, n, plan, digits):
    with Batch(bases, n) as bt:
        bt.set_plan(plan)
        for i, d in enumerate(digits):
            bt.put(i, d)
        bt.square(True, 1)
        bt.square(False, 2)
        bt.copy(1, 0)
        bt.init_multiplicand(1)
        bt.mul_into(0)
        return bt.get_all(0)


@pytest.mark.parametrize("n,plan,count,bmin,bmax", [
    (20, 304, 8, 1_100_000, 55_000_000),        # packed, 16-row columns
    (18, 204, 24, 1_100_000, 130_000_000),      # packed four-step
    (17, 203, 48, 1_100_000, 150_000_000),      # packed, 8-row columns
    (18, 103, 16, 1_000, 1_000_000_000),        # unpacked six-step, 2 and 3 primes
    (16, 3, 64, 1_000, 1_900_000_000),          # unpacked four-step, 8-row columns
    (12, 0, 320, 1_000, 1_900_000_000),         # single-CTA: 160 tests on each prime set
    (11, 0, 320, 1_000, 1_900_000_000),
])
def test_batch_matches_single_tests(oracle, n, plan, count, bmin, bmax):
    rng = np.random.default_rng(n * 100 + plan)
    if plan == 0:       # half on two primes, half on three (one launch per prime set)
        bases = [int(x) & ~1 for x in np.concatenate([rng.integers(bmin, 10_000_000, size=count // 2),
                                                      rng.integers(300_000_000, bmax, size=count - count // 2)])]
    else:
        bases = [int(x) & ~1 for x in rng.integers(bmin, bmax, size=count)]
    digits = [rng.integers(-(b // 2), b // 2 + 1, size=1 << n).astype(np.int32) for b in bases]
    got = run(bases, n, plan, digits)
    if plan == 0:
        with Batch(bases, n) as bt:
            w = bt.widths()
        assert np.count_nonzero(w == 2) >= 148 and np.count_nonzero(w == 3) >= 148
    for i in (0, count - 1):
        one = run([bases[i]], n, plan, [digits[i]])[0]
        assert np.array_equal(canon(got[i], bases[i]), canon(one, bases[i])), i
    o = oracle.OracleTransform(bases[0], n)
    o.setInt(digits[0])
    o.squareDup(True)
    o.squareDup(False)
    o.squareDup(False)
    o.copy(1, 0)
    o.mul(1)
    assert np.array_equal(canon(got[0], bases[0]), canon(o.getInt(), bases[0]))
