"""Fermat PRP driver over the engine: the caller side of the hot path.

``quick`` mirrors genefer::quick / prp / GL (src/genefer.h:736-748,
:479-552, :557-615) over a ``Transform`` (one squaring per call: the plain
path).  ``BatchPRP`` runs the same test for every test of a ``Batch``:
exponents are padded with leading zero bits to a common length (squaring the
initial 1 leaves it 1, and the Gerbicz-Li steps in the padded prefix multiply
d(t) by 1), so all tests share one block schedule and each Gerbicz-Li block
(B squarings + the d(t) update) is one CUDA graph replay.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import gint
from .exponent import B_GerbiczLi, bit, chunk_sum, exponent_words, prefix_words
from .transform import Batch, Transform


@dataclass
class Result:
    b: int
    n: int
    is_prp: bool
    res64: int
    old64: int
    gl_ok: bool


@dataclass
class Job:
    """One exponentiation 2^e mod b^(2^n)+1 as the PRP loop runs it: e is the
    test's exponent E = b^(2^n) (``full``) or its top ``bits`` bits
    (``prefix``), whose result is the state of the full test after ``bits``
    squarings (src/genefer.h:505-549 stopped early)."""
    b: int
    n: int
    words: np.ndarray
    nbits: int

    @classmethod
    def full(cls, b: int, n: int) -> "Job":
        w, nb = exponent_words(int(b), int(n))
        return cls(int(b), int(n), w, nb)

    def words_nbits(self):
        return self.words, self.nbits

    @classmethod
    def prefix(cls, b: int, n: int, bits: int) -> "Job":
        w, k, _ = prefix_words(int(b), int(n), int(bits))
        return cls(int(b), int(n), w, k)


# ------------------------------------------------------------------ one test

def prp(t: Transform, words: np.ndarray, nbits: int, B: int) -> None:
    """genefer::prp without checkpoints (src/genefer.h:479-552): reg0 = 2^E, reg1 = d(t)."""
    t.set(1)
    t.copy(1, 0)
    for i in range(nbits - 1, -1, -1):
        t.squareDup(bit(words, i))
        if (i % B == 0) and (i // B != 0):
            t.copy(2, 0)
            t.mul(1)
            t.copy(1, 0)
            t.copy(0, 2)


def GL(t: Transform, words: np.ndarray, nbits: int, B: int) -> bool:
    """genefer::GL (src/genefer.h:557-615)."""
    t.mul(1)
    t.copy(2, 0)
    t.copy(0, 1)
    for _ in range(B):
        t.squareDup(False)
    t.copy(1, 0)
    res = chunk_sum(words, nbits, B)
    t.set(1)
    for i in range(res.bit_length() - 1, -1, -1):
        t.squareDup(((res >> i) & 1) != 0)
    t.mul(1)
    h1 = gint.hash64(gint.unbalance(t.getInt(), t.b))
    t.copy(0, 2)
    h2 = gint.hash64(gint.unbalance(t.getInt(), t.b))
    return h1 == h2


def quick(t: Transform, B: Optional[int] = None) -> Result:
    """genefer::quick (src/genefer.h:736-748)."""
    words, nbits = exponent_words(t.b, t.n)
    if B is None:
        B = B_GerbiczLi(nbits)
    prp(t, words, nbits, B)
    is_prp, r64, o64 = gint.is_one(gint.unbalance(t.getInt(), t.b), t.b)
    ok = GL(t, words, nbits, B)
    return Result(t.b, t.n, is_prp, r64, o64, ok)


# ------------------------------------------------------------------ batches

def _pad(words: np.ndarray, nwords: int) -> np.ndarray:
    out = np.zeros(nwords, dtype=np.uint32)
    out[: words.size] = words
    return out


def _int_words(v: int) -> np.ndarray:
    nw = max(1, (int(v).bit_length() + 31) // 32)
    return np.frombuffer(int(v).to_bytes(4 * nw, "little"), dtype="<u4").astype(np.uint32)


def gl_validate(bt: Batch, B: int, res: Sequence[int]) -> np.ndarray:
    """genefer::GL (src/genefer.h:557-615) for every test of bt at once: reg0 =
    the residue r, reg1 = d(t), res[i] = sum of the B-bit chunks of test i's
    exponent; reg2 is overwritten.  Returns the per-test ok flags."""
    bt.init_multiplicand(1)
    bt.mul_into(0)                   # mul(1): r0 = r * d(t) = d(t+1)
    bt.copy(2, 0)
    bt.copy(0, 1)
    bt.square(False, B)              # d(t)^(2^B)
    bt.copy(1, 0)
    rbits = max(1, max(int(r).bit_length() for r in res))
    for i, r in enumerate(res):
        w = np.zeros((rbits + 31) // 32, dtype=np.uint32)
        rw = _int_words(r)
        w[: rw.size] = rw
        bt.set_exponent(i, w, rbits)
    bt.set(1)
    bt.square_exp(rbits)             # 2^res
    bt.init_multiplicand(1)
    bt.mul_into(0)                   # d(t)^(2^B) * 2^res
    a = bt.get_all(0)
    c = bt.get_all(2)
    ok = np.zeros(bt.count, dtype=bool)
    for i, b in enumerate(bt.bases):
        ok[i] = gint.hash64(gint.unbalance(a[i], int(b))) == gint.hash64(gint.unbalance(c[i], int(b)))
    return ok


class BatchPRP:
    """Fermat PRP tests of every test of a Batch with a common block length B.
    ``exps`` (one (words, nbits) per test) replaces the tests' exponents
    b^(2^n), e.g. by the prefixes of ``Job.prefix``."""

    def __init__(self, batch: Batch, B: Optional[int] = None, exps: Optional[Sequence] = None):
        self.batch = batch
        if exps is None:
            self.exps = [exponent_words(int(b), batch.n) for b in batch.bases]
        else:
            if len(exps) != batch.count:
                raise ValueError("one exponent per test")
            self.exps = [(np.asarray(w, dtype=np.uint32), int(nb)) for (w, nb) in exps]
        self.nbits = max(nb for _, nb in self.exps)
        self.B = int(B) if B else B_GerbiczLi(self.nbits)
        self._graph = None

    def load(self) -> None:
        """Uploads padded exponents; reg0 = 1, reg1 = d(t) = 1 (src/genefer.h:492-497)."""
        nw = (self.nbits + 31) // 32
        for i, (w, _) in enumerate(self.exps):
            self.batch.set_exponent(i, _pad(w, nw), self.nbits)
        self.batch.set(1)
        self.batch.copy(1, 0)

    def schedule(self) -> List[int]:
        """Block lengths: the first block ends at the highest multiple of B, then
        full blocks; a Gerbicz-Li step follows every block except the last."""
        i0 = self.nbits - 1
        first = i0 % self.B + 1
        blocks = [first]
        left = self.nbits - first
        while left > 0:
            blocks.append(self.B)
            left -= self.B
        return blocks

    def block_graph(self):
        if self._graph is None:
            bt, B = self.batch, self.B
            self._graph = bt.capture(lambda: (bt.square_exp(B), bt.gl_step()))
        return self._graph

    def run_prp(self, use_graph: bool = True) -> None:
        blocks = self.schedule()
        bt = self.batch
        for k, cnt in enumerate(blocks):
            last = (k == len(blocks) - 1)
            if last:
                bt.square_exp(cnt)
            elif use_graph and cnt == self.B:
                self.block_graph().launch()
            else:
                bt.square_exp(cnt)
                bt.gl_step()

    def validate(self) -> np.ndarray:
        """genefer::GL for every test (src/genefer.h:557-615); returns ok flags."""
        return gl_validate(self.batch, self.B, [chunk_sum(w, nb, self.B) for (w, nb) in self.exps])

    def results(self, validate: bool = True) -> List[Result]:
        """Residues of reg0 after run_prp (kept in ``canon``, canonical digits),
        then (optionally) the GL check, which overwrites the registers."""
        bt = self.batch
        r0 = bt.get_all(0)
        canon = [gint.unbalance(r0[i], int(b)) for i, b in enumerate(bt.bases)]
        self.canon = canon
        ok = self.validate() if validate else np.ones(bt.count, dtype=bool)
        out = []
        for i, b in enumerate(bt.bases):
            is_prp, r64, o64 = gint.is_one(canon[i], int(b))
            out.append(Result(int(b), bt.n, is_prp, r64, o64, bool(ok[i])))
        return out

    def run(self) -> List[Result]:
        self.load()
        self.run_prp()
        return self.results()


def quick_batch(bases: Sequence[int], n: int, B: Optional[int] = None, device: int = 0) -> List[Result]:
    with Batch(bases, n, num_regs=3, device=device) as bt:
        return BatchPRP(bt, B).run()
