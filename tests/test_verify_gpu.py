"""Periodic Gerbicz-Li verification with rollback (genefer22_b200.verify):
a full test reproduces the reference's residue, and a seeded bit flip written
into the device state is detected and undone."""
import numpy as np
import pytest

from genefer22_b200.verify import VerifiedPRP, flip_bit

pytestmark = pytest.mark.gpu

KAT = (23448336, 12, 0x81CFF004ACE85CAA)   # src/main.cpp:422


def test_verified_quick_kat():
    b, n, r64 = KAT
    v = VerifiedPRP(b, n, B=64, span=8)
    canon = v.run()
    assert v.residue(canon)[1] == r64
    assert v.stats.failures == 0 and v.stats.checks == v.stats.spans


def test_fault_detected_and_rolled_back():
    b, n, r64 = KAT
    rng = np.random.default_rng(1013)
    v = VerifiedPRP(b, n, B=64, span=8)
    at = int(rng.integers(0, v.nbits_pad))
    canon = v.run(fault=flip_bit(1013), fault_at=at)
    assert v.stats.fault_at == [at]
    assert v.stats.failures == 1 and v.stats.rollbacks == 1
    assert v.residue(canon)[1] == r64


def test_n20_fault_rollback_matches_clean_run():
    """Config of the n = 20 test: b seeded in [10^6, 5 10^7], checks every
    2000 squarings (B = 200, 10 blocks), one seeded fault; the state after the
    first spans equals the fault-free run."""
    rng = np.random.default_rng(1003)
    b = int(rng.integers(5 * 10**5, 25 * 10**6)) * 2
    clean = VerifiedPRP(b, 20, B=200, span=10)
    c0 = clean.run(max_spans=3)
    faulty = VerifiedPRP(b, 20, B=200, span=10)
    at = int(np.random.default_rng(1013).integers(2000, 4000))
    c1 = faulty.run(fault=flip_bit(7), fault_at=at, max_spans=3)
    assert clean.stats.failures == 0
    assert faulty.stats.failures == 1 and faulty.stats.fault_at == [at]
    assert np.array_equal(c0, c1)
