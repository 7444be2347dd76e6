"""Packed digits (plans 200 + lr): two base-b digits per coefficient of a
transform of N/2 points over four primes.  Results must equal the oracle's
(restated transformCPUi32) and the unpacked plans', digit for digit after
canonicalisation, through squarings, dup squarings, products, Gerbicz-Li
blocks replayed from graphs, plan switches with pending carries and slot
reassignment; bases outside the exact range are refused."""
import numpy as np
import pytest

from genefer22_b200 import Batch, GfcError, Transform, gint
from genefer22_b200 import genefer as gf
from genefer22_b200.exponent import words_to_int

pytestmark = pytest.mark.gpu

# largest even base of the exact packed range per n (the checks in packed_ok)
B_MAX = {16: 184393718, 17: 155056016, 18: 130386048}


def canon(d, b):
    return gint.unbalance(d, b)


def rand_digits(rng, b, N):
    return rng.integers(-(b // 2), b // 2 + 1, size=N).astype(np.int32)


@pytest.mark.parametrize("n,plan,b", [(12, 203, 2_000_002), (13, 204, 50_000_000), (14, 203, 2**20 + 2),
                                      (16, 204, 100_000_000), (16, 203, B_MAX[16]), (17, 204, 123_456_790),
                                      (18, 204, B_MAX[18])])
def test_packed_vs_oracle(oracle, n, plan, b):
    rng = np.random.default_rng(n + b % 97)
    t = Transform(b, n)
    t.batch.set_plan(plan)
    assert t.batch.plan() == plan and list(t.batch.widths()) == [4]
    o = oracle.OracleTransform(b, n)
    d = rand_digits(rng, b, 1 << n)
    t.setInt(d)
    o.setInt(d)
    for k in range(3):
        dup = (k == 1)
        t.squareDup(dup)
        o.squareDup(dup)
        g = t.getInt()
        assert np.abs(g).max() <= b // 2 + 1
        assert np.array_equal(canon(g, b), canon(o.getInt(), b)), f"square {k}"
    t.copy(1, 0); o.copy(1, 0)
    t.squareDup(False); o.squareDup(False)
    t.mul(1); o.mul(1)
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b)), "mul"
    t.copy(2, 0); o.copy(2, 0)
    t.initMultiplicand(2); o.initMultiplicand(2)
    t.squareDup(True); o.squareDup(True)
    t.mul(); o.mul()
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b)), "mul 2"


@pytest.mark.parametrize("n,plan,b", [(17, 303, 150_000_000), (18, 304, 100_000_002), (20, 305, 50_000_000),
                                      (21, 307, 77_000_000), (22, 305, 35_000_000), (23, 306, 25_000_002),
                                      (21, 303, 44_000_002), (21, 304, 40_000_000)])
def test_packed_six_step_vs_oracle(oracle, n, plan, b):
    """Packed digits with the six-step split of the half-length transform (from
    n = 21 the 2^3..2^5-row middle passes twist the rows)."""
    rng = np.random.default_rng(n + 7)
    t = Transform(b, n)
    t.batch.set_plan(plan)
    assert t.batch.plan() == plan
    o = oracle.OracleTransform(b, n)
    d = rand_digits(rng, b, 1 << n)
    t.setInt(d)
    o.setInt(d)
    for k, dup in enumerate((False, True, False)):
        t.squareDup(dup)
        o.squareDup(dup)
        g = t.getInt()
        assert np.abs(g).max() <= b // 2 + 1
        assert np.array_equal(canon(g, b), canon(o.getInt(), b)), f"square {k}"
    t.copy(1, 0); o.copy(1, 0)
    t.squareDup(False); o.squareDup(False)
    t.mul(1); o.mul(1)
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b)), "mul"
    t.copy(2, 0); o.copy(2, 0)
    t.initMultiplicand(2); o.initMultiplicand(2)
    t.squareDup(True); o.squareDup(True)
    t.mul(); o.mul()
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b)), "mul 2"


def test_range_refused():
    for b in (2**20 - 2, B_MAX[16] + 2):
        bt = Batch([b, 2_000_002], 16)
        with pytest.raises(GfcError):
            bt.set_plan(204)
        assert bt.plan() == 4 and list(bt.widths()) == [3 if b > 10**8 else 2, 2]
    bt = Batch([2_000_002], 16)
    bt.set_plan(204)
    with pytest.raises(GfcError):
        bt.assign(0, B_MAX[16] + 2)


def _blocks(bases, n, plan, B, nblk, exps):
    bt = Batch(bases, n)
    bt.set_plan(plan)
    r = gf.BatchPRP(bt, B=B, exps=exps)
    r.load()
    bt.square_exp(r.schedule()[0])
    bt.gl_step()
    g = r.block_graph()
    for _ in range(nblk):
        g.launch()
    out = (bt.get_pos(), bt.get_all(0), bt.get_all(1))
    r._graph = None
    bt.close()
    return out


@pytest.mark.parametrize("n,plan", [(16, 204), (15, 203)])
def test_packed_graph_blocks_match_unpacked(n, plan):
    rng = np.random.default_rng(n)
    bases = [int(x) & ~1 for x in rng.integers(1_100_000, 100_000_000, size=24)]
    B = 20
    exps = [gf.Job.prefix(b, n, 4 * B + (i % 5)).words_nbits() for i, b in enumerate(bases)]
    got = _blocks(bases, n, plan, B, 2, exps)
    ref = _blocks(bases, n, 4 if n == 16 else 3, B, 2, exps)
    assert np.array_equal(got[0], ref[0])
    for i, b in enumerate(bases):
        assert np.array_equal(canon(got[1][i], b), canon(ref[1][i], b)), i
        assert np.array_equal(canon(got[2][i], b), canon(ref[2][i], b)), i


@pytest.mark.parametrize("n,plan,ref,count", [(21, 303, 8, 5), (21, 304, 8, 5), (21, 305, 8, 4), (22, 304, 9, 3),
                                              (22, 305, 9, 3)])
def test_twisted_packed_blocks_match_four_step(n, plan, ref, count):
    """Batches on twisted six-step packed plans (two tests per row CTA, every
    row at table base 1) against the unpacked four-step plan, which has no
    middle pass: Gerbicz-Li blocks with exponents of different lengths, so that
    tests drop out at different squarings of the last block and row CTAs run
    pairs with one test left (and, with an odd count, a lone last test)."""
    rng = np.random.default_rng(n + plan)
    bases = [int(x) & ~1 for x in rng.integers(1_100_000, 30_000_000, size=count)]
    B = 20
    exps = [gf.Job.prefix(b, n, 4 * B + (i % 5)).words_nbits() for i, b in enumerate(bases)]
    got = _blocks(bases, n, plan, B, 2, exps)
    want = _blocks(bases, n, ref, B, 2, exps)
    assert np.array_equal(got[0], want[0])
    for i, b in enumerate(bases):
        assert np.array_equal(canon(got[1][i], b), canon(want[1][i], b)), i
        assert np.array_equal(canon(got[2][i], b), canon(want[2][i], b)), i


@pytest.mark.parametrize("n,count", [(17, 2), (17, 4), (18, 2)])
def test_small_packed_batches_match_unpacked(n, count):
    """Packed batches of a few tests: at n = 17 their row CTAs run one test's row
    each (a pair per CTA would halve a grid of 128-256 CTAs), at n = 18 (rows
    of 8192 points) two tests' rows per CTA; Gerbicz-Li blocks against the
    unpacked four-step plan."""
    rng = np.random.default_rng(n * 10 + count)
    bases = [int(x) & ~1 for x in rng.integers(1_100_000, 100_000_000, size=count)]
    B = 20
    exps = [gf.Job.prefix(b, n, 4 * B + (i % 5)).words_nbits() for i, b in enumerate(bases)]
    got = _blocks(bases, n, 204, B, 2, exps)
    want = _blocks(bases, n, 4 if n == 17 else 5, B, 2, exps)
    assert np.array_equal(got[0], want[0])
    for i, b in enumerate(bases):
        assert np.array_equal(canon(got[1][i], b), canon(want[1][i], b)), i
        assert np.array_equal(canon(got[2][i], b), canon(want[2][i], b)), i


@pytest.mark.parametrize("n,count,plan", [(20, 1, 303), (20, 2, 304), (21, 1, 305), (21, 3, 304), (22, 1, 305),
                                          (22, 2, 306), (23, 2, 306)])
def test_packed_default_plans_by_count(n, count, plan):
    """A new packed batch starts on the plan measured fastest for its size and
    number of tests."""
    bases = [20_000_002 + 2 * i for i in range(count)]
    with Batch(bases, n) as bt:
        assert bt.plan() == plan


def test_plan_switch_with_pending_carries(oracle):
    """Carries left pending by one plan are absorbed before the next takes over."""
    n, b = 16, 60_000_002
    rng = np.random.default_rng(5)
    bt = Batch([b, 3_000_002], n)
    d = [rand_digits(rng, b, 1 << n), rand_digits(rng, 3_000_002, 1 << n)]
    bt.put(0, d[0]); bt.put(1, d[1])
    bt.set_plan(204)
    bt.square(True, 2)
    bt.set_plan(4)
    bt.square(False, 1)
    bt.set_plan(204)
    bt.square(False, 1)
    for i, bb in enumerate((b, 3_000_002)):
        o = oracle.OracleTransform(bb, n)
        o.setInt(d[i])
        for dup in (True, True, False, False):
            o.squareDup(dup)
        assert np.array_equal(canon(bt.get(i), bb), canon(o.getInt(), bb)), i


def test_packed_finished_test_and_assign(oracle):
    n = 16
    jobs = [gf.Job.prefix(1_500_002, n, 30), gf.Job.prefix(99_999_998, n, 80)]
    bt = Batch([j.b for j in jobs], n)
    bt.set_plan(204)
    for i, j in enumerate(jobs):
        bt.set_exponent(i, j.words, j.nbits)
    bt.set(1)
    bt.copy(1, 0)
    bt.square_exp(50)
    bt.gl_step()
    bt.square_exp(40)
    for i, j in enumerate(jobs):
        o = oracle.OracleTransform(j.b, n)
        o.set(1)
        e = words_to_int(j.words)
        for k in range(j.nbits - 1, -1, -1):
            o.squareDup(bool((e >> k) & 1))
        assert np.array_equal(canon(bt.get(i, 0), j.b), canon(o.getInt(), j.b)), i
    # a new base in slot 0, squared with the packed kernels
    bt.assign(0, 77_777_778)
    rng = np.random.default_rng(9)
    dd = rand_digits(rng, 77_777_778, 1 << n)
    bt.put(0, dd)
    bt.square(True, 2)
    o = oracle.OracleTransform(77_777_778, n)
    o.setInt(dd)
    o.squareDup(True); o.squareDup(True)
    assert np.array_equal(canon(bt.get(0), 77_777_778), canon(o.getInt(), 77_777_778))


def test_packed_quick_residue():
    """A full test through the packed plan gives genefer's residue (the n = 12
    quick test of src/main.cpp:417-425 uses b = 10^9, beyond the packed range,
    so the reference residue here is the unpacked plan's)."""
    b, n = 2_000_002, 12
    t1 = Transform(b, n)
    r1 = gf.quick(t1)
    t2 = Transform(b, n)
    t2.batch.set_plan(203)
    r2 = gf.quick(t2)
    assert r2 == r1 and r2.gl_ok


@pytest.mark.parametrize("n,plan", [(16, 203), (16, 204), (20, 304)])
def test_packed_extreme_states(oracle, n, plan):
    """Digits at the resting bound +-(b/2 + 1) at the largest packed base: the
    half-length convolution reaches (N/2) ((b/2+1)(b+1))^2, next to the exact
    range of the four primes, and the carry window its largest values."""
    b = {16: B_MAX[16], 20: 55_000_000}[n]
    N = 1 << n
    h = b // 2 + 1
    states = [np.full(N, h, np.int32), np.full(N, -h, np.int32),
              np.where(np.arange(N) % 2 == 0, h, -h).astype(np.int32),
              np.where((np.arange(N) // 2) % 2 == 0, h, -h).astype(np.int32)]
    for d in states:
        bt = Batch([b], n)
        bt.set_plan(plan)
        bt.put(0, d)
        o = oracle.OracleTransform(b, n)
        o.setInt(canon(d, b))
        for dup in (False, True):
            bt.square(dup, 1)
            o.squareDup(dup)
            got = bt.get(0)
            assert np.abs(got).max() <= b // 2 + 1
            assert np.array_equal(canon(got, b), canon(o.getInt(), b)), (int(d[0]), int(d[1]), dup)
        bt.close()
