"""The integer identities the squaring kernels rely on, restated with Python
integers (CPU only; the kernels themselves are checked against the oracle by
the GPU tests):

* the Shoup product by a table root (gf_arith.cuh, shoup_mul): for a 31-bit
  prime p, a < 2^32 and w < p with q = floor(w 2^32 / p), a w - h p with
  h = floor(a q / 2^32) lies in [0, 2p), below 2^32, and is a w mod p;
* the packed CRT (crt_garner4, crt_window_g): the top-down test on Garner's
  mixed-radix digits decides V > M/2, and with the top digit a4 - p4 when it
  does, f V = sum_{j<5} U_j b^j for the base-b limbs of f p1, f p1 p2,
  f p1 p2 p3, with |U_j| and every window position inside the stated bounds;
* the fused CRT + carry of prime sets 0 and 1 (crt_carry<SET>): one 64-bit
  division by b and per-test constants give the balanced digit and the carry
  of f V + c exactly;
* the absorption of a segment's carry into the next 16 digits (absorb,
  absorb5): it fits for every carry the engine produces, keeps the value and
  leaves every digit within b/2 + 1 (the resting bound the exact ranges
  assume).
"""
import math

import numpy as np
import pytest

P31 = (127 * 2**24 + 1, 63 * 2**25 + 1, 15 * 2**27 + 1)                 # prime set 1
P2 = (127 * 2**24 + 1, 63 * 2**25 + 1, 249 * 2**23 + 1, 15 * 2**27 + 1)  # prime set 2 (packed)
M2 = P2[0] * P2[1] * P2[2] * P2[3]


def shoup(a, w, p):
    q = (w << 32) // p
    h = (a * q) >> 32
    return a * w - h * p


@pytest.mark.parametrize("p", sorted(set(P31 + P2)))
def test_shoup_product_range(p):
    rng = np.random.default_rng(p % 1000)
    cases = [(2**32 - 1, p - 1), (2**32 - 1, 1), (0, p - 1), (p - 1, p - 1), (p, p - 1)]
    cases += [(int(a), int(w)) for a, w in zip(rng.integers(0, 2**32, 4000, dtype=np.uint64),
                                              rng.integers(0, p, 4000, dtype=np.uint64))]
    for a, w in cases:
        t = shoup(a, w, p)
        assert 0 <= t < 2 * p < 2**32
        assert t % p == (a * w) % p


def garner4(v):
    """Mixed-radix digits of 0 <= v < M2 (what crt_garner4 computes from the
    residues v mod p_k)."""
    p1, p2, p3, p4 = P2
    x = [v % p for p in P2]
    a1 = x[0]
    a2 = (x[1] - a1) * pow(p1, -1, p2) % p2
    a3 = (x[2] - a1 - p1 * a2) * pow(p1 * p2, -1, p3) % p3
    a4 = (x[3] - a1 - p1 * a2 - p1 * p2 * a3) * pow(p1 * p2 * p3, -1, p4) % p4
    return a1, a2, a3, a4


def top_down_z(a1, a2, a3, a4):
    """crt_garner4's test of V > M/2 from the top digit down."""
    p1, p2, p3, p4 = P2
    low = a2 * p1 + a1
    rest_hi = a3 > (p3 - 1) // 2 or (a3 == (p3 - 1) // 2 and low > (p1 * p2) // 2)
    return a4 > (p4 - 1) // 2 or (a4 == (p4 - 1) // 2 and rest_hi)


def limbs(w, b, count):
    out = []
    for _ in range(count):
        out.append(w % b)
        w //= b
    assert w == 0
    return out


def window_terms(digits, z, f, b):
    """U_0..U_4 of crt_window_g for mixed-radix digits, flag z and f = 1, 2."""
    p1, p2, p3, p4 = P2
    a1, a2, a3, a4 = digits
    A4 = a4 - (p4 if z else 0)
    w1, w2, w3 = limbs(f * p1, b, 2), limbs(f * p1 * p2, b, 4), limbs(f * p1 * p2 * p3, b, 5)
    return [f * a1 + a2 * w1[0] + a3 * w2[0] + A4 * w3[0],
            a2 * w1[1] + a3 * w2[1] + A4 * w3[1],
            a3 * w2[2] + A4 * w3[2],
            a3 * w2[3] + A4 * w3[3],
            A4 * w3[4]]


def boundary_values():
    half = M2 // 2
    return [0, 1, half - 1, half, half + 1, M2 - 1, M2 - 2, (M2 - 1) // 2, P2[0] * P2[1] * P2[2] * ((P2[3] - 1) // 2)]


def test_top_down_test_is_v_above_half_m():
    rng = np.random.default_rng(5)
    vals = boundary_values() + [int.from_bytes(rng.bytes(16), "little") % M2 for _ in range(3000)]
    for v in vals:
        assert top_down_z(*garner4(v)) == (v > M2 // 2), v


@pytest.mark.parametrize("b", [2**20, 2**20 + 2, 3_000_002, 2**24, 100_000_000, 2**28 - 2])
def test_centred_window_expansion(b):
    rng = np.random.default_rng(b % 997)
    vals = boundary_values() + [int.from_bytes(rng.bytes(16), "little") % M2 for _ in range(1500)]
    for v in vals:
        d = garner4(v)
        z = top_down_z(*d)
        vc = v - M2 if z else v                       # the centred value, |vc| <= M/2
        for f in (1, 2):
            U = window_terms(d, z, f, b)
            assert sum(u * b**j for j, u in enumerate(U)) == f * vc


@pytest.mark.parametrize("b", [2**20, 2**22, 2**24 + 2, 2**26, 2**28 - 2])
def test_window_bounds(b):
    """Worst case over the digit ranges: each U_j at its stated bound, every
    window position (U_j of at most three coefficients, j = p - 2i) below
    2^61.4, so that carry_wide (|s| < 2^62) covers it with the carry added."""
    p1, p2, p3, p4 = P2
    worst = [0.0] * 5
    for f in (1, 2):
        for a4, z in ((p4 - 1, False), (0, True), ((p4 - 1) // 2, True)):
            U = window_terms((p1 - 1, p2 - 1, p3 - 1, a4), z, f, b)
            for j, u in enumerate(U):
                worst[j] = max(worst[j], math.log2(abs(u)) if u else 0.0)
    bounds = (60.6, 60.6, 60.0, 59.1, 45.0)
    for j in range(5):
        assert worst[j] < bounds[j], (j, worst[j])
    even = math.log2(2**worst[0] + 2**worst[2] + 2**worst[4])
    odd = math.log2(2**worst[1] + 2**worst[3])
    carry = max(even, odd) - math.log2(b)             # the digit before's carry into a position
    assert math.log2(2**max(even, odd) + 2**carry) < 61.4 < 62


# ---- the fused CRT + carry of prime sets 0 and 1 (gf_arith.cuh crt_carry<SET>)

P0 = (125 * 2**25 + 1, 243 * 2**24 + 1)
MASK = 2**64 - 1


def carry_constants(b, primes):
    """carry_constants() of the host code: T is the top Garner weight."""
    T = primes[0] if len(primes) == 2 else primes[0] * primes[1]
    M = math.prod(primes)
    k = (2**56 + b - 1) // b
    return dict(b=b, h=b // 2, binv=MASK // b, k=k, kb=k * b,
                q=[(f * T) // b for f in (1, 2)], r=[(f * T) % b for f in (1, 2)],
                mq=[((f * M) // b) & MASK for f in (1, 2)], mr=[(f * M) % b for f in (1, 2)])


def divb64(n, K):
    assert 0 <= n <= MASK
    q = (n * K["binv"]) >> 64
    r = n - q * K["b"]
    if r >= K["b"]:
        q, r = q + 1, r - K["b"]
    assert 0 <= r < K["b"]
    return q, r


def crt_carry(x, dup, K, c, primes):
    """The kernel's arithmetic (uint64 wrap-around as on the device)."""
    if len(primes) == 2:
        p1, p2 = primes
        a_top = (x[1] - x[0]) * pow(p1, -1, p2) % p2
        low = x[0]
        z = a_top * p1 + x[0] > (p1 * p2) // 2
    else:
        p1, p2, p3 = primes
        a2 = (x[1] - x[0]) * pow(p1, -1, p2) % p2
        a_top = (x[2] - x[0] - p1 * a2) * pow(p1 * p2, -1, p3) % p3
        low = a2 * p1 + x[0]
        z = a_top > (p3 - 1) // 2 or (a_top == (p3 - 1) // 2 and low > (p1 * p2) // 2)
    U = (low << dup) + K["r"][dup] * a_top + K["h"] + ((K["b"] - K["mr"][dup]) if z else 0)
    assert U <= MASK
    qv, rv = divb64((U + (c & MASK) + K["kb"]) & MASK, K)
    cout = (qv + K["q"][dup] * a_top - ((K["mq"][dup] + 1) if z else 0) - K["k"]) & MASK
    cout = cout - 2**64 if cout >= 2**63 else cout
    return rv - K["h"], cout


@pytest.mark.parametrize("primes", [P0, P31], ids=["set0", "set1"])
@pytest.mark.parametrize("b", [8, 1_000, 65_538, 22_000_000, 1_000_000_000, 2**31 - 2])
def test_fused_crt_carry_is_exact(primes, b):
    """digit + b * carry_out = f V_c + carry_in with the digit in [-b/2, b - b/2)
    and V_c the centred CRT value, for carries up to 2^54 in magnitude and
    every product coefficient the engine can form: |V_c| <= N (b/2 + 1)^2 with
    N <= 2^23, inside M/2 (the width rule picks the prime set that way; the
    carry out then stays far below 2^63, which makes the quotient assembled
    modulo 2^64 exact)."""
    M = math.prod(primes)
    K = carry_constants(b, primes)
    bound = min(M // 2, 2**23 * (b // 2 + 1) ** 2)
    rng = np.random.default_rng(b % 1009 + len(primes))
    vcs = [0, 1, -1, bound, -bound, bound - 1, -(bound - 1)] + \
          [int.from_bytes(rng.bytes(16), "little") % (2 * bound + 1) - bound for _ in range(800)]
    cs = [0, 1, -1, 2**54, -2**54] + [int(c) for c in rng.integers(-2**54, 2**54, 800)]
    for i, vc in enumerate(vcs):
        v = vc % M
        x = [v % p for p in primes]
        assert (v - M if v > M // 2 else v) == vc
        for dup in (0, 1):
            c = cs[(i * 7 + dup) % len(cs)]
            d, cout = crt_carry(x, dup, K, c, primes)
            assert -(b // 2) <= d < b - b // 2
            assert d + b * cout == (dup + 1) * vc + c, (v, dup, c)


# ---- carry absorption into a 16-digit segment (gf_kernels.cuh absorb, gf_arith.cuh absorb5)

SEG = 16


def carry_balanced(s, b):
    """carry_small / carry_wide: the balanced digit of s and floor((s + b/2) / b)."""
    h = b // 2
    q = (s + h) // b
    return s + h - q * b - h, q


def absorb(dg, c, b):
    """absorb<D>: reduce while |c| > 1, then leave the last +-1 in the next
    digit unreduced; False if the carry did not fit."""
    dg = list(dg)
    for k in range(len(dg)):
        if c == 0:
            break
        if abs(c) > 1:
            dg[k], c = carry_balanced(dg[k] + c, b)
        else:
            dg[k] += c
            c = 0
    return c == 0, dg


def absorb5(dg, cin, b):
    """absorb5<D>: a packed segment carry (cin[k] at digit k, k < 5)."""
    dg = list(dg)
    q, done = 0, False
    for k in range(len(dg)):
        if done:
            continue
        if k >= 5 and -1 <= q <= 1:
            dg[k] += q
            q, done = 0, True
            continue
        dg[k], q = carry_balanced(dg[k] + (cin[k] if k < 5 else 0) + q, b)
    return done or q == 0, dg


def value(dg, b):
    return sum(d * b**k for k, d in enumerate(dg))


@pytest.mark.parametrize("b", [8, 10, 1024, 65_538, 22_000_000, 1_000_000_000, 2**31 - 2])
def test_absorb_segment_carry(b):
    """The carry out of a segment (at most the largest product coefficient,
    2^23 (b/2 + 1)^2 times 2 for a doubled square, over b, plus one) fits in
    the next segment, the value is kept, and every digit ends within b/2 + 1."""
    h = b // 2
    cmax = (2 * 2**23 * (h + 1) ** 2) // b + 1
    rng = np.random.default_rng(b % 1013)
    for _ in range(400):
        dg = [int(x) for x in rng.integers(-h, b - h, SEG)]
        c = int(rng.integers(-cmax, cmax + 1)) if _ > 3 else (cmax, -cmax, 1, -1)[_]
        ok, out = absorb(dg, c, b)
        assert ok, (b, c)
        assert value(out, b) == value(dg, b) + c
        assert max(abs(d) for d in out) <= h + 1


@pytest.mark.parametrize("b", [2**20, 2**20 + 2, 5_000_002, 2**24, 100_000_000, 2**28 - 2])
def test_absorb5_packed_segment_carry(b):
    """A packed segment carry (five window positions below 2^62 in magnitude)
    fits in the next 16-digit segment, the value is kept, and every digit ends
    within b/2 + 1."""
    h = b // 2
    lim = int(2**61.4)
    rng = np.random.default_rng(b % 1019)
    for i in range(400):
        dg = [int(x) for x in rng.integers(-h, b - h, SEG)]
        if i < 4:
            cin = [(lim, -lim)[i % 2]] * 5 if i < 2 else [(lim, -lim)[i % 2]] * 3 + [0, 0]
        else:
            cin = [int.from_bytes(rng.bytes(8), "little") % (2 * lim + 1) - lim for _ in range(5)]
        ok, out = absorb5(dg, cin, b)
        assert ok, (b, cin)
        assert value(out, b) == value(dg, b) + value(cin, b)
        assert max(abs(d) for d in out) <= h + 1


@pytest.mark.parametrize("b", [2, 3, 8, 1023, 2**20 + 7, 2**28 - 2, 2**31 - 1])
def test_barrett_division_by_b(b):
    """divb64: q = mulhi(n, floor((2^64 - 1) / b)) is floor(n / b) or one less
    for every n < 2^64, so one compare completes it."""
    binv = MASK // b
    rng = np.random.default_rng(b % 97)
    ns = [0, 1, b - 1, b, MASK, MASK - 1, MASK - b, (MASK // b) * b, (MASK // b) * b - 1] + \
         [int.from_bytes(rng.bytes(8), "little") for _ in range(3000)]
    for n in ns:
        q = (n * binv) >> 64
        assert n // b - q in (0, 1), (n, b)
