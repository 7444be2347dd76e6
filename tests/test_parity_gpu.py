"""Parity of the CUDA engine with the CPU oracle (restated transformCPUi32):
canonical residues must be identical after every operation."""
import numpy as np
import pytest

from genefer22_b200 import Batch, Transform, gint
from genefer22_b200 import genefer as gf

pytestmark = pytest.mark.gpu


def canon(d, b):
    return gint.unbalance(d, b)


def rand_digits(rng, b, N):
    return rng.integers(-(b // 2), b // 2 + 1, size=N).astype(np.int32)


def check_ops(oracle, b, n, plan=None, seed=0, steps=4):
    rng = np.random.default_rng(seed)
    t = Transform(b, n)
    if plan is not None:
        t.batch.set_plan(plan)
    o = oracle.OracleTransform(b, n)
    d = rand_digits(rng, b, 1 << n)
    t.setInt(d)
    o.setInt(d)
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b))
    for k in range(steps):
        dup = (k % 2 == 1)
        t.squareDup(dup)
        o.squareDup(dup)
        g = t.getInt()
        assert np.abs(g).max() <= b // 2 + 1
        assert np.array_equal(canon(g, b), canon(o.getInt(), b)), f"square {k}"
    # Gerbicz-Li style multiply: reg1 = r; square; r0 *= reg1
    t.copy(1, 0); o.copy(1, 0)
    t.squareDup(False); o.squareDup(False)
    t.mul(1); o.mul(1)
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b)), "mul"
    t.copy(2, 0); o.copy(2, 0)
    t.initMultiplicand(2); o.initMultiplicand(2)
    t.mul(); o.mul()
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b)), "mul 2"


# b values exercise both RNS widths: small b -> 2 primes, large b -> 3 primes
SMALL_B = 2 * 10**6
LARGE_B = 2 * 10**9 - 2


@pytest.mark.parametrize("n", [10, 11, 12, 13, 14])
@pytest.mark.parametrize("b", [SMALL_B, LARGE_B])
def test_single_cta_plan(oracle, n, b):
    check_ops(oracle, b, n, plan=0, seed=n)


@pytest.mark.parametrize("n", [12, 13, 14])
def test_lone_small_test_defaults_to_cluster(n):
    """A lone test at n = 12..14 squares on the cluster plan (eight SMs) by
    default, a wide batch on the single-CTA plan (one SM per test)."""
    assert Transform(SMALL_B, n).batch.plan() == 1
    assert Batch([SMALL_B] * 64, n).plan() == 0


@pytest.mark.parametrize("n,lr", [(11, 3), (14, 3), (12, 4), (13, 5), (14, 6), (12, 3), (15, 3), (15, 7), (16, 4), (16, 8),
                                  (17, 9), (18, 10)])
@pytest.mark.parametrize("b", [SMALL_B, LARGE_B])
def test_four_step_plan(oracle, n, lr, b):
    check_ops(oracle, b, n, plan=lr, seed=100 + n + lr, steps=3)


# six-step plans 100 + lr2: a 16-point column pass, a 2^lr2-point middle pass, rows
@pytest.mark.parametrize("n,plan", [(16, 103), (16, 104), (17, 104), (18, 105), (19, 106), (20, 107), (21, 105)])
@pytest.mark.parametrize("b", [SMALL_B, LARGE_B])
def test_six_step_plan(oracle, n, plan, b):
    check_ops(oracle, b, n, plan=plan, seed=200 + n + plan, steps=3)


# Six-step plans whose middle pass twists the rows (the row-pass root tables of one direction
# reach 32 MB: 8 B per point on the two-prime set, 24 B on the three-prime set), with 2^4 and
# 2^5-row middle passes; the two-prime base at n = 21 keeps the plain rows.
@pytest.mark.parametrize("n,plan", [(21, 104), (22, 105)])
@pytest.mark.parametrize("b", [SMALL_B // 4, LARGE_B])
def test_twisted_six_step_plans(oracle, n, plan, b):
    check_ops(oracle, b, n, plan=plan, seed=400 + n + plan, steps=3)


# The default unpacked plans of the two largest sizes (106 at n = 22, 107 at n = 23), which
# serve every base outside the packed-digit range (b < 2^20, or above the packed limit):
# squarings, dup squarings, mul by a register and initMultiplicand + mul against the oracle.
# Both bases lie outside the packed range (below 2^20, above 2^28), so they take these plans by
# default.
@pytest.mark.parametrize("n,plan", [(22, 106), (23, 107)])
@pytest.mark.parametrize("b", [SMALL_B // 4, LARGE_B])
def test_six_step_default_plans_largest_sizes(oracle, n, plan, b):
    assert Transform(b, n).batch.plan() == plan
    check_ops(oracle, b, n, plan=plan, seed=300 + n, steps=3)


def test_width_choice():
    # unpacked: 2 primes while N (b/2+1)^2 < P1 P2 / 2, else 3; packed digits
    # (the default from n = 16 for bases in the packed range): 4
    assert Transform(SMALL_B, 12).width() == 2
    assert Transform(LARGE_B, 12).width() == 3
    for b, w in ((22_000_000, 2), (23_500_000, 3)):
        t = Transform(b, 16)
        assert t.width() == 4 and t.batch.plan() == 203
        t.batch.set_plan(4)
        assert t.width() == w


@pytest.mark.parametrize("b", [8, 10, 1024, 1026, 65536 + 2])
def test_small_bases(oracle, b):
    check_ops(oracle, b, 12, seed=b)


def test_width_boundary(oracle):
    n = 13
    N = 1 << n
    M = (125 * 2**25 + 1) * (243 * 2**24 + 1)
    # largest even b with N (b/2+1)^2 < M/2
    h = int(((M // 2) // N) ** 0.5) + 2
    while N * (h + 1) ** 2 >= M // 2:
        h -= 1
    b_hi = 2 * h
    assert Transform(b_hi, n).width() == 2
    assert Transform(b_hi + 2, n).width() == 3
    for b in (b_hi, b_hi + 2):
        check_ops(oracle, b, n, seed=b % 1000)


def test_extreme_states(oracle):
    """All digits at +-b/2 (maximum convolution size) and the zero state."""
    b, n = 10**9, 12
    for fill in (b // 2, -(b // 2)):
        t, o = Transform(b, n), oracle.OracleTransform(b, n)
        d = np.full(1 << n, fill, np.int32)
        t.setInt(d); o.setInt(d)
        for k in range(3):
            t.squareDup(k == 1); o.squareDup(k == 1)
            assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b))
    t = Transform(b, n)
    t.setInt(np.zeros(1 << n, np.int32))
    t.squareDup(True)
    assert not np.any(t.getInt())


def test_set_and_context(oracle):
    b, n = 1_000_000, 12
    t = Transform(b, n)
    t.set(3)
    t.squareDup(False)
    z = t.getInt()
    assert z[0] == 9 and not np.any(z[1:])
    ctx = t.saveContext(2)
    t.squareDup(True)
    assert t.readContext(ctx, 2)
    assert np.array_equal(t.getInt(), z)
    assert not t.readContext(ctx[:-4], 2)


# src/main.cpp:417-425: quick-test residues at the 2-prime limits, 10^9, 2*10^9
KATS = {(33160956, 11): 0x9E2D51DA6C7C3F54, (64611980, 11): 0x6E2E19E3382BC8E8,
        (1000000000, 11): 0x43C6CC5326E5C77F, (2000000000, 11): 0x1A16EAEE2487902D,
        (23448336, 12): 0x81CFF004ACE85CAA, (45687570, 12): 0x6C3EA0FBFFEE2C34,
        (1000000000, 12): 0x4E43A5B93273C649, (2000000000, 12): 0xE5F3EA34F6C68EBD}


@pytest.mark.parametrize("b,n", [(23448336, 12), (2000000000, 12)])
def test_quick_kat_plain(b, n):
    r = gf.quick(Transform(b, n))
    assert r.res64 == KATS[(b, n)]
    assert r.gl_ok and not r.is_prp


def test_quick_kat_batch():
    for n in (11, 12):
        bases = [b for (b, nn) in KATS if nn == n]
        res = gf.quick_batch(bases, n)
        for r in res:
            assert r.res64 == KATS[(r.b, n)], hex(r.res64)
            assert r.gl_ok


def test_batch_matches_single(oracle):
    rng = np.random.default_rng(11)
    n = 12
    bases = [int(x) // 2 * 2 for x in rng.integers(1024, 2 * 10**9, size=6)] + [SMALL_B, 4096]
    bt = Batch(bases, n)
    digs = [rand_digits(rng, b, 1 << n) for b in bases]
    for i, d in enumerate(digs):
        bt.put(i, d)
    bt.square(True, 3)
    got = bt.get_all(0)
    for i, b in enumerate(bases):
        o = oracle.OracleTransform(b, n)
        o.setInt(digs[i])
        for _ in range(3):
            o.squareDup(True)
        assert np.array_equal(canon(got[i], b), canon(o.getInt(), b))


@pytest.mark.parametrize("plan", [0, 4])
def test_batch_exponent_graph(oracle, plan):
    """square_exp + gl_step recorded in a CUDA graph equals the driver loop."""
    n = 12
    bases = [1_000_002, 50_000_000, 1_999_999_998]
    bt = Batch(bases, n)
    bt.set_plan(plan)
    runner = gf.BatchPRP(bt, B=64)
    runner.load()
    bt.square_exp(5)
    g = runner.block_graph()
    g.launch()
    g.launch()
    pos = bt.get_pos()
    got0, got1 = bt.get_all(0), bt.get_all(1)
    for i, b in enumerate(bases):
        E = runner.exps[i]
        words = np.zeros((runner.nbits + 31) // 32, np.uint32)
        words[: E[0].size] = E[0]
        o = oracle.OracleTransform(b, n)
        o.set(1); o.copy(1, 0)
        i0 = runner.nbits - 1
        for k in range(5 + 2 * 64):
            idx = i0 - k
            o.squareDup(bool((int(words[idx >> 5]) >> (idx & 31)) & 1))
            if k == 4 or k == 68 or k == 132:
                if k != 4:
                    o.copy(2, 0); o.mul(1); o.copy(1, 0); o.copy(0, 2)
        assert pos[i] == i0 - (5 + 128)
        assert np.array_equal(canon(got0[i], b), canon(o.getInt(), b))
        o.copy(0, 1)
        assert np.array_equal(canon(got1[i], b), canon(o.getInt(), b))


@pytest.mark.parametrize("plan", [None, 4])
@pytest.mark.parametrize("b", [SMALL_B, LARGE_B, 1024])
def test_square_mul(oracle, b, plan):
    """transform::squareMul (prime mode): r <- a r^2 for small, large and negative a."""
    n = 12
    rng = np.random.default_rng(b % 97)
    t, o = Transform(b, n), oracle.OracleTransform(b, n)
    if plan is not None:
        t.batch.set_plan(plan)
    d = rand_digits(rng, b, 1 << n)
    t.setInt(d); o.setInt(d)
    for a in (3, 1, 2, -1, 0x7fffffff, -0x80000000 + 1, 12345, 0, 7):
        if a == 0:
            t.setInt(d); o.setInt(d)
            continue
        t.squareMul(a); o.squareMul(a)
        g = t.getInt()
        assert np.abs(g).max() <= b // 2 + 1
        assert np.array_equal(canon(g, b), canon(o.getInt(), b)), f"a={a}"


@pytest.mark.parametrize("b", [10, 1026, LARGE_B])
def test_digit_range_checked_on_load(b):
    """gfc_batch_set_zi / gfc_batch_set_all accept |d| <= b/2 + 1 and refuse one
    digit beyond it (either sign, any position) with GFC_ERR_ARG, leaving the
    register as it was."""
    from genefer22_b200._lib import GfcError
    n, lim = 12, b // 2 + 1
    rng = np.random.default_rng(b)
    with Batch([b, b], n) as bt:
        ok = rand_digits(rng, b, 1 << n)
        ok[0], ok[-1], ok[7] = lim, -lim, lim
        bt.put(0, ok)
        assert np.array_equal(bt.get(0), ok)
        for pos, v in ((5, lim + 1), ((1 << n) - 1, -lim - 1), (0, 2**31 - 1), (3, -2**31)):
            bad = ok.copy()
            bad[pos] = v
            with pytest.raises(GfcError):
                bt.put(0, bad)
            both = np.stack([ok, bad])
            with pytest.raises(GfcError):
                bt.put_all(both)
            assert np.array_equal(bt.get(0), ok)
        bt.put_all(np.stack([ok, ok]))
        assert np.array_equal(bt.get_all(0)[1], ok)
