"""genefer's deterministic primality test of N = b^(2^n) + 1 (mode "prime",
src/genefer.h:1101-1217) over the engine.

Brillhart, Lehmer and Selfridge, Theorem 1: N is prime if for every prime p
dividing N - 1 = b^(2^n) there is a base a with a^(N-1) = 1 and
a^((N-1)/p) != 1 (mod N).  For each base the engine computes
a^((N-1)/b) = a^(b^(2^n - 1)) with one ``squareMul`` per exponent bit
(x <- x^2 a or x^2), then ``power`` raises it to b / p and to p for every
prime p | b whose condition is still open.  The first base is the smallest
odd a2 >= 3 whose Kronecker symbol genefer's test finds to be -1; the next
ones are 2, 3, 4, ... skipping a2 and squares (src/genefer.h:1126-1141).

A context file (src/genefer.h:278-366; version, base index k, bit index,
elapsed and total seconds, the conditions met, the transform's registers 0
and 1, CRC) lets a stopped test resume.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

from . import gint
from .exponent import exponent_words, words_to_int
from .proof import CONTEXT_VERSION_GPU, KIND_NTT3, FileError, GFile, power


def powmod(a: int, e: int, m: int) -> int:
    """arith.h:13-25 as written: right-to-left square-and-multiply followed
    by one more product with the last square, so that for e = 2^k it returns
    a^(2^(k+1)) mod m.  Restated unchanged because it decides which first
    base the test uses."""
    r, t, i = 1, a % m, e
    while i != 1:
        if i % 2 != 0:
            r = (r * t) % m
        t = (t * t) % m
        i //= 2
    r = (r * t) % m
    return (r * t) % m


def kronecker(x: int, y: int) -> int:
    """Kronecker symbol (x / y) (arith.h:27-53)."""
    tab = (0, 1, 0, -1, 0, -1, 0, 1)
    if (x & 1) == 0 and (y & 1) == 0:
        return 0
    a, b = x, y
    v = 0
    while (b & 1) == 0:
        b >>= 1
        v = 1 - v
    if (v & 1) == 0:
        k = 1
    elif a == 0:
        k = 0
    else:
        k = tab[a & 7]
    while True:
        if a == 0:
            if b > 1:
                return 0
            if b == 1:
                return k
        v = 0
        while (a & 1) == 0:
            a >>= 1
            v = 1 - v
        if (v & 1) != 0 and b != 0 and tab[b & 7] == -1:
            k = -k
        if (a & b & 2) != 0:
            k = -k
        a, b = b % a, a


def prime_factors(n: int) -> List[int]:
    """Distinct prime factors in increasing order (arith.h:55-76)."""
    p, r = [], n
    if r % 2 == 0:
        while r % 2 == 0:
            r //= 2
        p.append(2)
    d = 3
    while r != 1:
        if r % d == 0:
            while r % d == 0:
                r //= d
            p.append(d)
        d += 2
    return p


def first_base(b: int, n: int) -> int:
    """genefer's a2 (src/genefer.h:1126-1129)."""
    a2 = 3
    while kronecker((powmod(b % a2, 1 << n, a2) + 1) % a2, a2) != -1:
        a2 += 2
    return a2


def bases(b: int, n: int):
    """The bases in the order genefer tries them: a2, then k = 2, 3, ...
    without a2 and without squares."""
    a2 = first_base(b, n)
    k = 1
    while True:
        if k != a2 and (k == 1 or math.isqrt(k) ** 2 != k):
            yield k, (a2 if k == 1 else k)
        k += 1


@dataclass
class PrimeResult:
    is_prime: Optional[bool]           # None: stopped before a decision
    bases: List[int] = field(default_factory=list)
    cond: List[bool] = field(default_factory=list)
    factors: List[int] = field(default_factory=list)


def _save(path: str, t, k: int, i: int, elapsed: float, total: float, cond: List[bool]):
    new, old = path + ".new", path + ".old"
    with GFile(new, "wb") as f:
        f.write_i32(CONTEXT_VERSION_GPU)
        f.write_i32(k)
        f.write_i32(i)
        f.write_f64(elapsed)
        f.write_f64(total)
        f.write_i32(len(cond))
        for c in cond:
            f.write_i32(1 if c else 0)
        f.write_i32(KIND_NTT3)
        f.write(t.saveContext(2))
        f.write_crc32()
    if os.path.exists(old):
        os.remove(old)
    if os.path.exists(path):
        os.rename(path, old)
    os.rename(new, path)


def _load_one(path: str, t, ncond: int) -> Optional[Tuple[int, int, float, float, List[bool]]]:
    if not os.path.exists(path):
        return None
    try:
        with GFile(path, "rb") as f:
            if f.read_i32() != CONTEXT_VERSION_GPU:
                return None
            k, i = f.read_i32(), f.read_i32()
            elapsed, total = f.read_f64(), f.read_f64()
            nc = f.read_i32()
            if nc != ncond:
                return None
            cond = [f.read_i32() != 0 for _ in range(nc)]
            if f.read_i32() != KIND_NTT3:
                return None
            payload = f.read(t.contextSize(2))
            if not f.check_crc32():
                return None
    except FileError:
        return None
    if not t.readContext(payload, 2):
        return None
    return k, i, elapsed, total, cond


def prime(t, b: int, n: int, ctx: Optional[str] = None, save_every: int = 0,
          abort_at: Optional[Tuple[int, int]] = None) -> PrimeResult:
    """genefer::prime (src/genefer.h:1101-1217).  ``abort_at = (k, i)`` stops
    before bit i of base index k, saving the context, as genefer's
    quitting() does."""
    pf = prime_factors(b)
    w, _ = exponent_words(b, n)
    E = words_to_int(w) // b                     # b^(2^n - 1)
    i0 = E.bit_length() - 1
    cond = [False] * len(pf)
    found = None
    if ctx:
        found = _load_one(ctx, t, len(pf)) or _load_one(ctx + ".old", t, len(pf))
    rk = 1
    if found is not None:
        rk, ri, _, _, cond = found
    res = PrimeResult(None, [], cond, pf)
    for k, a in bases(b, n):
        if k < rk:
            continue
        if found is None:
            t.set(1)
        i_start = ri if found is not None else i0
        found = None
        for i in range(i_start, -1, -1):
            if ctx and ((abort_at is not None and (k, i) == tuple(abort_at))
                        or (save_every and i != i_start and i % save_every == 0)):
                _save(ctx, t, k, i, 0.0, 0.0, cond)
                if abort_at is not None and (k, i) == tuple(abort_at):
                    return res
            t.squareMul(a if (E >> i) & 1 else 1)
        t.copy(1, 0)
        res.bases.append(a)
        composite = False
        for j, p in enumerate(pf):
            if cond[j]:
                continue
            power(t, 1, b // p)                   # a^((N-1)/p)
            if not gint.is_one(gint.unbalance(t.getInt(), b), b)[0]:
                cond[j] = True
            power(t, 0, p)                        # a^(N-1)
            if not gint.is_one(gint.unbalance(t.getInt(), b), b)[0]:
                composite = True
                break
        if composite:
            res.is_prime = False
            return res
        if all(cond):
            res.is_prime = True
            return res
