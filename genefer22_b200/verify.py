"""Fermat PRP test with periodic Gerbicz-Li verification and rollback.

genefer checks Gerbicz-Li (GL) once, at the end of a test (src/genefer.h:557-615);
an error found there fails the whole test.  ``VerifiedPRP`` checks the GL
identity after every span of m blocks of B squarings and, on a mismatch,
returns to the last verified state and redoes the span, so a transient error
costs one span instead of the test.

With x_j the residue after block j (x_{j+1} = x_j^(2^B) 2^(e_{j+1}), e the
B-bit exponent chunk consumed by the block), a span from block s to s+m is
correct when

    D^(2^B) * 2^S * x_s == D * x_(s+m),   D = x_s x_(s+1) ... x_(s+m-1),
                                          S = e_(s+1) + ... + e_(s+m),

the telescoped form of the identity genefer verifies (there with m = all blocks
and D accumulated by the prp loop, src/genefer.h:529-535).  D is accumulated on
the device by the d(t) update; the check costs B squarings and four products.

Registers: 0 = x (running residue), 1 = D, 2 = x_s (last verified residue),
3, 4 = scratch.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import gint
from .exponent import exponent_words
from .transform import Batch

NUM_REGS = 5


@dataclass
class VerifyStats:
    spans: int = 0
    checks: int = 0
    failures: int = 0
    rollbacks: int = 0
    squarings: int = 0            # exponent squarings, redone ones included
    check_squarings: int = 0      # squarings spent in checks
    fault_at: List[int] = field(default_factory=list)


def _chunk(bits: np.ndarray, hi: int, B: int) -> int:
    """Value of the B exponent bits hi, hi-1, ..., hi-B+1 (bits: little-endian uint8 array)."""
    v = 0
    for i in range(hi, hi - B, -1):
        v = (v << 1) | int(bits[i])
    return v


class VerifiedPRP:
    """2^E mod b^(2^n)+1, E = b^(2^n), with a GL check every `span` blocks of B
    squarings.  `fault` is an optional callback (batch, squaring_index) used
    to inject an error into the device state once, for tests."""

    def __init__(self, b: int, n: int, B: int, span: int, device: int = 0):
        self.b, self.n, self.B, self.m = int(b), int(n), int(B), int(span)
        words, nbits = exponent_words(self.b, self.n)
        self.nbits_pad = ((nbits + self.B - 1) // self.B) * self.B
        nw = (self.nbits_pad + 31) // 32
        padded = np.zeros(nw, dtype=np.uint32)
        padded[: words.size] = words
        self.words = padded
        self.bits = np.unpackbits(padded.view(np.uint8), bitorder="little")
        self.batch = Batch([self.b], self.n, num_regs=NUM_REGS, device=device)
        self.stats = VerifyStats()
        if (1 << (self.m - 1)) > self.b // 2:
            raise ValueError("span too long for this base (2^(S >> B) < 2^m must fit in one digit)")

    # ---------------------------------------------------------------- helpers

    def _run_blocks(self, pos: int, nblocks: int, fault: Optional[Callable], fault_at: Optional[int]) -> int:
        """Blocks of B squarings from bit position pos; d(t) update after each
        block but the last.  Returns the new position."""
        bt, B = self.batch, self.B
        for k in range(nblocks):
            start = self.nbits_pad - 1 - pos       # index of the first squaring of this block
            if (fault is not None) and (fault_at is not None) and (start <= fault_at < start + B):
                first = fault_at - start
                bt.square_exp(first)
                fault(bt, fault_at)
                self.stats.fault_at.append(fault_at)
                bt.square_exp(B - first)
            else:
                bt.square_exp(B)
            self.stats.squarings += B
            pos -= B
            if k < nblocks - 1:
                bt.gl_step()
        return pos

    def _check(self, pos_start: int, nblocks: int) -> bool:
        """GL identity for the span that started at pos_start (regs 0..2 as above)."""
        bt, B = self.batch, self.B
        S = sum(_chunk(self.bits, pos_start - k * B, B) for k in range(nblocks))
        s_hi, s_lo = S >> B, S & ((1 << B) - 1)
        bt.init_multiplicand(1)
        bt.mul_into(3)                     # reg3 = D x_(s+m)
        bt.copy(4, 0)                      # keep x_(s+m)
        bt.set(1 << s_hi)
        bt.init_multiplicand(1)
        bt.mul_into(0)                     # 2^(S_hi) D
        for i in range(B - 1, -1, -1):
            bt.square(bool((s_lo >> i) & 1), 1)   # (2^(S_hi) D)^(2^B) 2^(S_lo) = D^(2^B) 2^S
        self.stats.check_squarings += B
        bt.init_multiplicand(2)
        bt.mul_into(0)                     # * x_s
        lhs = gint.unbalance(bt.get(0, 0), self.b)
        rhs = gint.unbalance(bt.get(0, 3), self.b)
        bt.copy(0, 4)                      # restore x_(s+m)
        self.stats.checks += 1
        return bool(np.array_equal(lhs, rhs))

    # ---------------------------------------------------------------- run

    def run(self, fault: Optional[Callable] = None, fault_at: Optional[int] = None,
            max_spans: Optional[int] = None) -> np.ndarray:
        """Runs the test (or its first max_spans spans) and returns the canonical
        digits of the residue."""
        bt = self.batch
        bt.set_exponent(0, self.words, self.nbits_pad)
        bt.set(1)
        bt.copy(2, 0)                      # x_s = 1
        bt.copy(1, 0)                      # D = x_s
        pos = self.nbits_pad - 1
        nblocks_total = self.nbits_pad // self.B
        done_blocks = 0
        injected = False
        while done_blocks < nblocks_total:
            if (max_spans is not None) and (self.stats.spans >= max_spans):
                break
            nb = min(self.m, nblocks_total - done_blocks)
            pos_s = pos
            use_fault = fault if not injected else None
            pos = self._run_blocks(pos, nb, use_fault, fault_at)
            if use_fault is not None and self.stats.fault_at:
                injected = True
            if self._check(pos_s, nb):
                bt.copy(2, 0)              # new verified x_s
                bt.copy(1, 0)              # D restarts at x_s
                done_blocks += nb
                self.stats.spans += 1
            else:                          # roll back to the last verified state
                self.stats.failures += 1
                self.stats.rollbacks += 1
                bt.copy(0, 2)
                bt.copy(1, 2)
                bt.set_pos([pos_s])
                pos = pos_s
        return gint.unbalance(bt.get(0, 0), self.b)

    def residue(self, canon: np.ndarray):
        """(isPrp, res64, old64) of canonical digits (gint::isOne)."""
        return gint.is_one(canon, self.b)


def flip_bit(seed: int) -> Callable:
    """A fault that flips one seeded bit of one seeded digit of register 0
    (written from the host into device memory, then re-balanced)."""
    rng = np.random.default_rng(seed)

    def fault(bt: Batch, squaring: int):
        d = bt.get(0, 0)
        i = int(rng.integers(0, d.size))
        bit = int(rng.integers(0, 20))
        d[i] ^= (1 << bit)
        bt.put(0, gint.balance(d, int(bt.bases[0])), 0)
    return fault
