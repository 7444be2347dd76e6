"""genefer's proof, server and check modes and its file formats, over the
engine.

* ``GFile``: genefer's ``file`` (src/file.h:66-161): bytes with a running
  CRC-32 (polynomial 0xEDB88320, the one zlib uses), closed by
  ``write_crc32`` / ``check_crc32`` (stored as ~crc ^ 0xa23777ac); GMP integers
  in ``mpz_out_raw`` format (4-byte big-endian signed byte count, then the
  magnitude big-endian), which genefer does not add to the CRC.
* ``write_gint`` / ``read_gint``: gint::write / read (src/gint.h:151-167):
  size, base, canonical digits.
* Context files (src/genefer.h:199-276): version (-1 for a GPU build), where
  (0: prp, 1: check), bit index, elapsed seconds, the transform's context,
  CRC; written to ``.new`` and renamed, the previous one kept as ``.old``.
* ``prp``: genefer::prp (src/genefer.h:478-552) with Gerbicz-Li updates, the
  Pietrzak-Li checkpoints copied to registers 3 + i / B_PL (fast
  checkpoints), and a context saved every ``save_every`` bits and at an
  abort, from which a later call resumes.
* ``PL``: proof generation (src/genefer.h:620-734), ``server``: proof
  verification and certificate (:770-885), ``check``: certificate check
  (:887-1099), ``proof``: prp + GL + PL (:750-766).

The transform is any object with genefer's transform interface (``set``,
``squareDup``, ``initMultiplicand``, ``mul``, ``copy``, ``getInt``,
``setInt``, and ``saveContext`` / ``readContext`` for context files): the
CUDA ``Transform`` in production.  Integers that genefer keeps in GMP (the
exponent, the proof weights w, the certificate exponent p2) are Python ints.
"""
from __future__ import annotations

import os
import struct
import time
import zlib
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

from . import gint
from .exponent import B_GerbiczLi

KIND_NTT3 = 7                  # transform::EKind::NTT3 (src/transform.h:45)
CONTEXT_VERSION_GPU = -1       # genefer's GPU build negates version 1 (src/genefer.h:206-210)


class FileError(RuntimeError):
    """A bad or truncated file (genefer's file::error)."""


class GFile:
    """genefer's ``file`` with its running CRC-32 (src/file.h:66-161)."""

    def __init__(self, path: str, mode: str):
        if mode not in ("rb", "wb"):
            raise ValueError("mode is 'rb' or 'wb'")
        self.path, self.mode = path, mode
        self._f = open(path, mode)
        self.crc = 0

    def close(self):
        if self._f is not None:
            self._f.close()
            self._f = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # raw bytes (CRC updated)
    def write(self, data: bytes):
        self._f.write(data)
        self.crc = zlib.crc32(data, self.crc)

    def read(self, size: int) -> bytes:
        data = self._f.read(size)
        self.crc = zlib.crc32(data, self.crc)
        if len(data) != size:
            raise FileError(f"{self.path}: failure of a read operation")
        return data

    def write_i32(self, v: int):
        self.write(struct.pack("<i", int(v)))

    def read_i32(self) -> int:
        return struct.unpack("<i", self.read(4))[0]

    def write_f64(self, v: float):
        self.write(struct.pack("<d", float(v)))

    def read_f64(self) -> float:
        return struct.unpack("<d", self.read(8))[0]

    # GMP integers: mpz_out_raw / mpz_inp_raw, outside the CRC (src/file.h:124-137)
    def write_mpz(self, v: int):
        v = int(v)
        mag = abs(v)
        nb = (mag.bit_length() + 7) // 8
        self._f.write(struct.pack(">i", -nb if v < 0 else nb) + mag.to_bytes(nb, "big"))

    def read_mpz(self) -> int:
        hdr = self._f.read(4)
        if len(hdr) != 4:
            raise FileError(f"{self.path}: failure of a read operation")
        nb = struct.unpack(">i", hdr)[0]
        data = self._f.read(abs(nb))
        if len(data) != abs(nb):
            raise FileError(f"{self.path}: failure of a read operation")
        v = int.from_bytes(data, "big")
        return -v if nb < 0 else v

    def write_crc32(self):
        self.write(struct.pack("<I", (~self.crc ^ 0xa23777ac) & 0xffffffff))

    def check_crc32(self) -> bool:
        expect = (~self.crc ^ 0xa23777ac) & 0xffffffff
        got = struct.unpack("<I", self.read(4))[0]
        return got == expect


def write_gint(f: GFile, digits: np.ndarray, b: int):
    """gint::write (src/gint.h:160-167): size, base, canonical digits."""
    d = np.ascontiguousarray(gint.unbalance(digits, b), dtype="<i4")
    f.write(struct.pack("<II", d.size, int(b)))
    f.write(d.tobytes())


def read_gint(f: GFile, size: int, b: int) -> np.ndarray:
    """gint::read (src/gint.h:151-158): the size and base must match."""
    s, base = struct.unpack("<II", f.read(8))
    if s != size or base != b:
        raise FileError(f"{f.path}: bad file")
    return np.frombuffer(f.read(4 * size), dtype="<i4").astype(np.int32)


def hash32(canon: np.ndarray) -> int:
    """gint::gethash32 (src/gint.h:221-225)."""
    h = gint.hash64(canon)
    return max(2, (h & 0xffffffff) ^ (h >> 32))


def B_PietrzakLi(esize: int, depth: int) -> int:
    """genefer::B_PietrzakLi (src/genefer.h:473-476)."""
    return ((int(esize) - 1) >> int(depth)) + 1


# ------------------------------------------------------------------ contexts

def save_context(path: str, t, where: int, i: int, elapsed: float, num_regs: int):
    """genefer::saveContext (src/genefer.h:245-276)."""
    new, old = path + ".new", path + ".old"
    with GFile(new, "wb") as f:
        f.write_i32(CONTEXT_VERSION_GPU)
        f.write_i32(where)
        f.write_i32(i)
        f.write_f64(elapsed)
        f.write_i32(KIND_NTT3)
        f.write(t.saveContext(num_regs))
        f.write_crc32()
    if os.path.exists(old):
        os.remove(old)
    if os.path.exists(path):
        os.rename(path, old)
    os.rename(new, path)


def _read_context_file(path: str, t, where: int, num_regs: int) -> Optional[Tuple[int, float]]:
    if not os.path.exists(path):
        return None
    try:
        with GFile(path, "rb") as f:
            if f.read_i32() != CONTEXT_VERSION_GPU or f.read_i32() != where:
                return None
            i = f.read_i32()
            elapsed = f.read_f64()
            if f.read_i32() != KIND_NTT3:
                return None
            payload = f.read(t.contextSize(num_regs))
            if not f.check_crc32():
                return None
    except FileError:
        return None
    if not t.readContext(payload, num_regs):
        return None
    return i, elapsed


def read_context(path: str, t, where: int, num_regs: int) -> Optional[Tuple[int, float]]:
    """genefer::readContext (src/genefer.h:199-243): the context file, else
    its ``.old`` copy; (bit index, elapsed seconds) or None."""
    r = _read_context_file(path, t, where, num_regs)
    if r is None:
        r = _read_context_file(path + ".old", t, where, num_regs)
    return r


# ------------------------------------------------------------------ powers

def power(t, reg: int, e: int):
    """r0 = r_reg^e (genefer::power / powerz, src/genefer.h:441-465)."""
    t.initMultiplicand(reg)
    t.set(1)
    e = int(e)
    if e == 0:
        return
    for i in range(e.bit_length() - 1, -1, -1):
        t.squareDup(False)
        if (e >> i) & 1:
            t.mul()


def _canon(t, b: int) -> np.ndarray:
    return gint.unbalance(t.getInt(), b)


def _bit(e: int, i: int) -> bool:
    return ((e >> i) & 1) != 0


# ------------------------------------------------------------------ prp with checkpoints

@dataclass
class Run:
    status: str                # "done" or "aborted"
    i: int                     # next bit to process (-1 when done)
    elapsed: float


def prp(t, E: int, B_GL: int, B_PL: int = 0, ctx: Optional[str] = None, save_every: int = 0,
        abort_at: Optional[int] = None) -> Run:
    """genefer::prp (src/genefer.h:478-552): reg0 = 2^E, reg1 = d(t); with
    B_PL, reg 3 + i / B_PL = the residue at bit i for i % B_PL == 0.  With a
    context path the run resumes from it and saves one every ``save_every``
    bits; ``abort_at`` stops before bit i as genefer's quitting() does (the
    context is saved)."""
    num_ctx = 0 if B_PL else 2
    found = read_context(ctx, t, 0, num_ctx) if ctx else None
    if found is None:
        t.set(1)
        t.copy(1, 0)
        i_start, base = E.bit_length() - 1, 0.0
    else:
        i_start, base = found
        if i_start == -1:
            return Run("done", -1, base)
    t0 = time.perf_counter()
    for i in range(i_start, -1, -1):
        if ctx and ((abort_at is not None and i == abort_at) or (save_every and i != i_start and i % save_every == 0)):
            save_context(ctx, t, 0, i, base + time.perf_counter() - t0, num_ctx)
            if abort_at is not None and i == abort_at:
                return Run("aborted", i, base + time.perf_counter() - t0)
        t.squareDup(_bit(E, i))
        if (i % B_GL == 0) and (i // B_GL != 0):
            t.copy(2, 0)
            t.mul(1)
            t.copy(1, 0)
            t.copy(0, 2)
        if B_PL and (i % B_PL == 0):
            t.copy(3 + i // B_PL, 0)
    elapsed = base + time.perf_counter() - t0
    if ctx:
        save_context(ctx, t, 0, -1, elapsed, num_ctx)
    return Run("done", -1, elapsed)


def GL(t, b: int, E: int, B_GL: int) -> bool:
    """genefer::GL (src/genefer.h:557-615)."""
    t.mul(1)
    t.copy(2, 0)
    t.copy(0, 1)
    for _ in range(B_GL):
        t.squareDup(False)
    t.copy(1, 0)
    res, e, mask = 0, E, (1 << B_GL) - 1
    while e:
        res += e & mask
        e >>= B_GL
    t.set(1)
    for i in range(res.bit_length() - 1, -1, -1):
        t.squareDup(_bit(res, i))
    t.mul(1)
    h1 = gint.hash64(_canon(t, b))
    t.copy(0, 2)
    h2 = gint.hash64(_canon(t, b))
    return h1 == h2


# ------------------------------------------------------------------ proof, server, check

def PL(t, b: int, depth: int, path: str) -> int:
    """Pietrzak-Li proof from the fast checkpoints in registers 3 .. 3 + 2^depth
    - 1 (src/genefer.h:620-734); writes the proof file, returns pkey."""
    L = 1 << depth
    with GFile(path, "wb") as f:
        f.write_i32(1)
        f.write_i32(depth)
        t.copy(0, 3)
        mu = _canon(t, b)
        write_gint(f, mu, b)
        q = hash32(mu)
        t.setInt(mu)
        power(t, 0, q)
        t.copy(2, 0)                                  # v1 = mu[0]^w[0]
        w = [0] * (L // 2)
        w[0] = q
        for k in range(1, depth + 1):
            i = 1 << (depth - k)
            t.copy(0, 3 + i)
            power(t, 0, w[0])                         # mu[k] = ckpt[i]^w[0]
            t.copy(1, 0)
            for j in range(i, L // 2, i):
                t.copy(0, 3 + i + 2 * j)
                power(t, 0, w[j])                     # mu[k] *= ckpt[i + 2j]^w[j]
                t.mul(1)
                t.copy(1, 0)
            mu = _canon(t, b)
            write_gint(f, mu, b)
            q = hash32(mu)
            power(t, 0, q)                            # v1 = v1 mu[k]^q
            t.mul(2)
            t.copy(2, 0)
            if i > 1:
                for j in range(0, L // 2, i):
                    w[i // 2 + j] = w[j] * q
        f.write_crc32()
    t.copy(0, 2)
    return gint.hash64(_canon(t, b))


@dataclass
class ProofResult:
    is_prp: bool
    res64: int
    old64: int
    gl_ok: bool
    pkey: int


def proof(t, b: int, n: int, depth: int, path: str, E: Optional[int] = None, ctx: Optional[str] = None,
          save_every: int = 0) -> ProofResult:
    """genefer::proof (src/genefer.h:750-766) with fast checkpoints: t needs
    3 + 2^depth registers."""
    from .exponent import exponent_words, words_to_int
    if E is None:
        w, _ = exponent_words(b, n)
        E = words_to_int(w)
    esize = E.bit_length()
    B_GL, B_PL = B_GerbiczLi(esize), B_PietrzakLi(esize, depth)
    r = prp(t, E, B_GL, B_PL, ctx=ctx, save_every=save_every)
    if r.status != "done":
        raise RuntimeError("prp did not finish")
    is_prp, r64, o64 = gint.is_one(_canon(t, b), b)
    ok = GL(t, b, E, B_GL)
    pkey = PL(t, b, depth, path)
    return ProofResult(is_prp, r64, o64, ok, pkey)


@dataclass
class ServerResult:
    is_prp: bool
    res64: int
    old64: int
    pkey: int
    ckey: int


def server(t, b: int, n: int, proof_path: str, cert_path: str, rnd: Tuple[int, int, int],
           E: Optional[int] = None) -> ServerResult:
    """genefer::server (src/genefer.h:770-885): reads a proof, recomputes
    pkey and writes the certificate.  rnd = (rnd1, rnd2, rnd3), which genefer
    draws from std::rand in [2, 64), [16, 256), [4, 65536)."""
    from .exponent import exponent_words, words_to_int
    if E is None:
        w, _ = exponent_words(b, n)
        E = words_to_int(w)
    N = 1 << n
    rnd1, rnd2, rnd3 = (int(x) for x in rnd)
    with GFile(proof_path, "rb") as f:
        f.read_i32()                                  # version
        depth = f.read_i32()
        L = 1 << depth
        B = B_PietrzakLi(E.bit_length(), depth)
        w = [0] * L
        mu = read_gint(f, N, b)
        is_prp, r64, o64 = gint.is_one(mu, b)
        q = hash32(mu)
        w[0] = q
        t.setInt(mu)
        power(t, 0, q)
        t.copy(1, 0)                                  # v1 = mu[0]^w[0]
        t.set(1)
        t.copy(2, 0)                                  # v2 = 1
        for k in range(1, depth + 1):
            mu = read_gint(f, N, b)
            q = hash32(mu)
            t.setInt(mu)
            t.copy(3, 0)
            power(t, 0, q)                            # v1 = v1 mu[k]^q
            t.mul(1)
            t.copy(1, 0)
            power(t, 2, q)                            # v2 = v2^q mu[k]
            t.mul(3)
            t.copy(2, 0)
            i = 1 << (depth - k)
            for j in range(0, L, 2 * i):
                w[i + j] = w[j] * q
        if not f.check_crc32():
            raise FileError(f"{proof_path}: bad file (crc32)")
    t.copy(0, 1)
    pkey = gint.hash64(_canon(t, b))
    p2, e = 0, E
    for i in range(L):
        p2 += (e & ((1 << B) - 1)) * w[i]
        e >>= B
    tt = rnd1 << B
    if p2 > tt:
        p2 -= tt
        t.set(2)
        power(t, 0, rnd1)
        t.mul(2)
        t.copy(2, 0)
    power(t, 1, rnd2)
    t.copy(1, 0)
    t.set(2)
    power(t, 0, rnd3)
    t.mul(1)
    ckey = gint.hash64(_canon(t, b))
    power(t, 2, rnd2)
    v = _canon(t, b)
    p2 = p2 * rnd2 + rnd3
    with GFile(cert_path, "wb") as f:
        f.write_i32(1)
        f.write_i32(B)
        write_gint(f, v, b)
        f.write_mpz(p2)
        f.write_crc32()
    return ServerResult(is_prp, r64, o64, pkey, ckey)


def check(t, b: int, n: int, cert_path: str, ctx: Optional[str] = None, save_every: int = 0,
          abort_at: Optional[int] = None) -> Optional[int]:
    """genefer::check (src/genefer.h:887-1099): v2^(2^B) 2^p2 with Gerbicz
    (the squarings of v2) and Gerbicz-Li (2^p2) error checks; returns ckey,
    None if a check failed, or raises on a bad certificate.  With a context
    path the run resumes from it; ``abort_at`` stops before bit i."""
    N = 1 << n
    with GFile(cert_path, "rb") as f:
        f.read_i32()
        B = f.read_i32()
        v2 = read_gint(f, N, b)
        p2 = f.read_mpz()
        if not f.check_crc32():
            raise FileError(f"{cert_path}: bad file (crc32)")
    p2size = p2.bit_length()
    L, GLb = B_GerbiczLi(B), B_GerbiczLi(p2size)
    found = read_context(ctx, t, 1, 3) if ctx else None
    ri, base = found if found is not None else (0, 0.0)
    t0 = time.perf_counter()
    i0 = p2size + B - 1

    def stop(i):
        if ctx and ((abort_at is not None and i == abort_at) or (save_every and i % save_every == 0)):
            save_context(ctx, t, 1, i, base + time.perf_counter() - t0, 3)
            return abort_at is not None and i == abort_at
        return False

    if found is None or ri >= p2size:
        if found is None:
            t.setInt(v2)
            t.copy(1, 0)                              # d(t) = u(0)
        for i in range(ri if found is not None else i0, p2size - 1, -1):
            if stop(i):
                return None
            j = i0 - i
            if (j % L == 0) and (j != 0):
                t.copy(2, 0)
                t.mul(1)
                t.copy(1, 0)
                t.copy(0, 2)
            t.squareDup(False)
        t.copy(2, 0)                                  # v2^(2^B)
        if B % L != 0:
            for _ in range(L - (B % L)):
                t.squareDup(False)
        t.mul(1)
        t.copy(3, 0)                                  # d(t+1)
        t.copy(0, 1)
        for _ in range(L):
            t.squareDup(False)
        t.copy(1, 0)                                  # d(t)^(2^L)
        t.setInt(v2)
        t.mul(1)                                      # u(0) d(t)^(2^L)
        h1 = gint.hash64(_canon(t, b))
        t.copy(0, 3)
        h2 = gint.hash64(_canon(t, b))
        if h1 != h2:
            return None
    if found is None or ri >= p2size:
        t.set(1)
        t.copy(1, 0)
        i_start = p2size - 1
    else:
        i_start = min(ri, p2size - 1)
    for i in range(i_start, -1, -1):
        if stop(i):
            return None
        t.squareDup(_bit(p2, i))
        if (i % GLb == 0) and (i // GLb != 0):
            t.copy(3, 0)
            t.mul(1)
            t.copy(1, 0)
            t.copy(0, 3)
    t.copy(3, 0)
    t.mul(2)                                          # v1' = v2 2^p2
    ckey = gint.hash64(_canon(t, b))
    t.copy(0, 3)
    t.mul(1)
    t.copy(2, 0)                                      # d(t+1)
    t.copy(0, 1)
    for _ in range(GLb):
        t.squareDup(False)
    t.copy(1, 0)
    res, e = 0, p2
    while e:
        res += e & ((1 << GLb) - 1)
        e >>= GLb
    t.set(1)
    for i in range(res.bit_length() - 1, -1, -1):
        t.squareDup(_bit(res, i))
    t.mul(1)
    h1 = gint.hash64(_canon(t, b))
    t.copy(0, 2)
    h2 = gint.hash64(_canon(t, b))
    if h1 != h2:
        return None
    return ckey
