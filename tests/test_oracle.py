"""Pins the CPU oracle (oracle/gf_oracle.c, a restatement of
transformCPUi32 + gint) against the residues quoted in the reference's own
sources and against the reference transform compiled from its sources."""
import numpy as np
import pytest

# design/rns.cpp:596-603 (b = 10^9): res64 of 2^(b^(2^n)) mod b^(2^n)+1
RNS_KATS = {5: 0x7da127b73585c207, 6: 0xc37bd72acdea47e1, 7: 0xcfa99a35cc4a7179, 8: 0x280cd7361db156d7,
            9: 0x0629e1b97daab9df, 10: 0x9983e7718a7d7a4d}

# src/main.cpp:417-420 (n = 11) and :422-425 (n = 12)
MAIN_KATS_11 = {33160956: 0x9E2D51DA6C7C3F54, 64611980: 0x6E2E19E3382BC8E8,
                1000000000: 0x43C6CC5326E5C77F, 2000000000: 0x1A16EAEE2487902D}
MAIN_KATS_12 = {23448336: 0x81CFF004ACE85CAA, 45687570: 0x6C3EA0FBFFEE2C34,
                1000000000: 0x4E43A5B93273C649, 2000000000: 0xE5F3EA34F6C68EBD}


@pytest.mark.parametrize("n", sorted(RNS_KATS))
def test_oracle_rns_kats(oracle, n):
    is_prp, res64, _, ok = oracle.quick(oracle.OracleTransform(10**9, n), 10**9, n)
    assert res64 == RNS_KATS[n]
    assert ok and not is_prp


@pytest.mark.slow
@pytest.mark.parametrize("b", sorted(MAIN_KATS_11))
def test_oracle_main_kats_n11(oracle, b):
    is_prp, res64, _, ok = oracle.quick(oracle.OracleTransform(b, 11), b, 11)
    assert res64 == MAIN_KATS_11[b] and ok


def test_oracle_main_kat_n11_one(oracle):
    b = 33160956
    _, res64, _, ok = oracle.quick(oracle.OracleTransform(b, 11), b, 11)
    assert res64 == MAIN_KATS_11[b] and ok


def test_oracle_gl_detects_fault(oracle):
    """A +1 injected into the state makes Gerbicz-Li fail (the reference's
    commented add1() hook, src/transform.h:248-255, src/genefer.h:526-527)."""
    b, n = 10**9, 8
    t = oracle.OracleTransform(b, n)
    E = oracle.exponent(b, n)
    B = oracle.B_GerbiczLi(E.bit_length())
    t.set(1)
    t.copy(1, 0)
    for i in range(E.bit_length() - 1, -1, -1):
        t.squareDup(((E >> i) & 1) != 0)
        if i == E.bit_length() // 2:
            d = t.getInt()
            d[0] += 1
            t.setInt(d)
        if (i % B == 0) and (i // B != 0):
            t.copy(2, 0); t.mul(1); t.copy(1, 0); t.copy(0, 2)
    assert not oracle.GL(t, E, B, b)


def test_gint_roundtrip(oracle):
    rng = np.random.default_rng(7)
    b, N = 123456, 1 << 10
    d = rng.integers(-(2**31) // 4, 2**31 // 4, size=N).astype(np.int32)
    c = oracle.unbalance(d, b)
    assert c.min() >= 0 and c.max() < b
    bal = oracle.balance(d, b)
    assert np.all(bal > -b // 2 - 1) and np.all(bal <= b // 2)
    assert np.array_equal(oracle.unbalance(bal, b), c)


needs_ref = pytest.mark.skipif("not __import__('gf_oracle').ref_available()", reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("n", [6, 9, 12])
def test_oracle_matches_reference_raw(oracle, n):
    """The restatement's raw RNS state equals the reference's, bit for bit."""
    rng = np.random.default_rng(100 + n)
    b = int(rng.integers(1024, 2 * 10**9)) // 2 * 2
    o, r = oracle.OracleTransform(b, n), oracle.RefTransform(b, n)
    d = rng.integers(-(b // 2), b // 2, size=1 << n).astype(np.int32)
    o.setInt(d)
    r.setInt(d)
    for k in range(4):
        o.squareDup(k % 2 == 1)
        r.squareDup(k % 2 == 1)
        assert np.array_equal(o.raw(), r.raw())
    o.copy(1, 0); r.copy(1, 0)
    o.squareDup(False); r.squareDup(False)
    o.mul(1); r.mul(1)
    assert np.array_equal(o.raw(), r.raw())
    assert np.array_equal(o.getInt(), r.getInt())


@needs_ref
def test_reference_rns_kat(oracle):
    _, res64, _, ok = oracle.quick(oracle.RefTransform(10**9, 9), 10**9, 9)
    assert res64 == RNS_KATS[9] and ok


@needs_ref
def test_oracle_square_mul_matches_reference(oracle):
    rng = np.random.default_rng(77)
    b, n = 1_000_000_006, 10
    o, r = oracle.OracleTransform(b, n), oracle.RefTransform(b, n)
    d = rng.integers(-(b // 2), b // 2, size=1 << n).astype(np.int32)
    o.setInt(d); r.setInt(d)
    for a in (3, 5, 123456789, 2):
        o.squareMul(a); r.squareMul(a)
        assert np.array_equal(o.raw(), r.raw())
