"""The six-step twist of the row pass, on the CPU in plain integers.

The row pass of a six-step squaring transforms row k of the R x C matrix the
middle pass leaves with the roots of table base R + k.  The middle pass twists
instead: it multiplies element c of row k by nu_k^c = H[m][c] G[c]^brev(q)
(k = m 2^lr2 + q, H and G as k_twist in gf_kernels.cuh writes them), after
which every row transforms with the roots of base 1 (the first C entries of
the table) and the inverse is untwisted by the inverse factors.  These tests
check that identity on small transforms for the primes of every prime set,
forward and inverse, exactly as the CUDA kernels compose it.
"""
import random

import pytest

PRIMES = [125 * 2**25 + 1, 243 * 2**24 + 1, 127 * 2**24 + 1, 63 * 2**25 + 1, 15 * 2**27 + 1, 249 * 2**23 + 1]


def brev(x: int, bits: int) -> int:
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def primitive_root(p: int) -> int:
    f, m, d = [], p - 1, 2
    while d * d <= m:
        if m % d == 0:
            f.append(d)
            while m % d == 0:
                m //= d
        d += 1
    if m > 1:
        f.append(m)
    g = 2
    while any(pow(g, (p - 1) // q, p) == 1 for q in f):
        g += 1
    return g


def psi_of(p: int, n: int) -> int:
    return pow(primitive_root(p), (p - 1) // (2 << n), p)


def block_fwd(x, base, tw, p):
    """Cooley-Tukey stages of one block (len(x) points) at table base `base`:
    local stage t uses entry (base << t) + sb for sub-block sb."""
    x = list(x)
    L = len(x).bit_length() - 1
    for t in range(L):
        half = len(x) >> (t + 1)
        for sb in range(1 << t):
            w = tw[(base << t) + sb]
            for i in range(half):
                j = sb * 2 * half + i
                a, b = x[j], x[j + half] * w % p
                x[j], x[j + half] = (a + b) % p, (a - b) % p
    return x


def block_inv(x, base, twi, p):
    """Gentleman-Sande stages in reverse order (no normalisation)."""
    x = list(x)
    L = len(x).bit_length() - 1
    for t in reversed(range(L)):
        half = len(x) >> (t + 1)
        for sb in range(1 << t):
            w = twi[(base << t) + sb]
            for i in range(half):
                j = sb * 2 * half + i
                a, b = x[j], x[j + half]
                x[j], x[j + half] = (a + b) % p, (a - b) * w % p
    return x


def twist_tables(p, n, lr, inverse):
    """H[m][c] and G[c] as k_twist computes them (normal form here)."""
    psi = psi_of(p, n)
    if inverse:
        psi = pow(psi, -1, p)
    C, two_n = 1 << (n - lr), 2 << n
    H = [[pow(psi, (c * (2 * brev(m, 4) + 1) + two_n - ((c << lr) % two_n)) % two_n, p) for c in range(C)]
         for m in range(16)]
    G = [pow(psi, (32 * c) % two_n, p) for c in range(C)]
    return H, G


@pytest.mark.parametrize("p", PRIMES)
@pytest.mark.parametrize("n,lr2", [(10, 2), (11, 3), (12, 4)])
def test_twisted_rows_equal_rows_at_their_base(p, n, lr2):
    N, lr = 1 << n, 4 + lr2
    R, C = 1 << lr, 1 << (n - lr)
    psi = psi_of(p, n)
    assert pow(psi, N, p) == p - 1
    tw = [pow(psi, brev(i, n), p) for i in range(N)]
    twi = [pow(psi, -brev(i, n), p) for i in range(N)]
    Hf, Gf = twist_tables(p, n, lr, False)
    Hi, Gi = twist_tables(p, n, lr, True)
    rng = random.Random(p ^ n)
    for k in rng.sample(range(R), 6) + [0, R - 1]:
        m, q = k >> lr2, k & ((1 << lr2) - 1)
        row = [rng.randrange(p) for _ in range(C)]
        f = [Hf[m][c] * pow(Gf[c], brev(q, lr2), p) % p for c in range(C)]
        fi = [Hi[m][c] * pow(Gi[c], brev(q, lr2), p) % p for c in range(C)]
        assert all(a * b % p == 1 for a, b in zip(f, fi))
        # forward: the row at base R + k == the twisted row at base 1
        ref = block_fwd(row, R + k, tw, p)
        got = block_fwd([x * fc % p for x, fc in zip(row, f)], 1, tw, p)
        assert got == ref
        # inverse: base R + k == base 1, then untwist
        ref_i = block_inv(ref, R + k, twi, p)
        got_i = [x * fc % p for x, fc in zip(block_inv(ref, 1, twi, p), fi)]
        assert got_i == ref_i
        assert ref_i == [x * C % p for x in row]
