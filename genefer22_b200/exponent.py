"""Exponent E = b^(2^n) of the Fermat PRP test (src/genefer.h:1476) and the
Gerbicz-Li block schedule (src/genefer.h:467-471, :557-615).

genefer computes E with GMP; this module calls the same library
(libgmp.so.10) through ctypes when it is present and falls back to Python
integers otherwise.  Only the exponent's bits reach the device.
"""
from __future__ import annotations

import ctypes
import ctypes.util
from typing import Tuple

import numpy as np

_gmp = None
_gmp_tried = False


def _load_gmp():
    global _gmp, _gmp_tried
    if _gmp_tried:
        return _gmp
    _gmp_tried = True
    for name in ("libgmp.so.10", ctypes.util.find_library("gmp")):
        if not name:
            continue
        try:
            g = ctypes.CDLL(name)
        except OSError:
            continue
        g.__gmpz_init.argtypes = [ctypes.c_void_p]
        g.__gmpz_clear.argtypes = [ctypes.c_void_p]
        g.__gmpz_ui_pow_ui.argtypes = [ctypes.c_void_p, ctypes.c_ulong, ctypes.c_ulong]
        g.__gmpz_sizeinbase.restype = ctypes.c_size_t
        g.__gmpz_sizeinbase.argtypes = [ctypes.c_void_p, ctypes.c_int]
        g.__gmpz_export.restype = ctypes.c_void_p
        g.__gmpz_export.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t), ctypes.c_int, ctypes.c_size_t,
                                    ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p]
        _gmp = g
        break
    return _gmp


def exponent_words(b: int, n: int) -> Tuple[np.ndarray, int]:
    """E = b^(2^n) as little-endian uint32 words and its bit length."""
    g = _load_gmp()
    if g is not None:
        z = ctypes.create_string_buffer(32)   # mpz_t (16 bytes), padded
        g.__gmpz_init(z)
        try:
            g.__gmpz_ui_pow_ui(z, b, 1 << n)
            nbits = int(g.__gmpz_sizeinbase(z, 2))
            words = np.zeros((nbits + 31) // 32, dtype=np.uint32)
            cnt = ctypes.c_size_t(0)
            g.__gmpz_export(words.ctypes.data, ctypes.byref(cnt), -1, 4, 0, 0, z)
        finally:
            g.__gmpz_clear(z)
        return words, nbits
    E = pow(int(b), 1 << n)
    nbits = E.bit_length()
    nw = (nbits + 31) // 32
    return np.frombuffer(E.to_bytes(4 * nw, "little"), dtype="<u4").astype(np.uint32), nbits


def words_to_int(words: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(words, dtype="<u4").tobytes(), "little")


def bit(words: np.ndarray, i: int) -> bool:
    return bool((int(words[i >> 5]) >> (i & 31)) & 1)


def B_GerbiczLi(esize: int) -> int:
    """genefer::B_GerbiczLi (src/genefer.h:467-471)."""
    L = 2 << ((int(esize).bit_length() - 1) // 2)
    return (int(esize) - 1) // L + 1


def chunk_sum(words: np.ndarray, nbits: int, B: int) -> int:
    """Sum of the B-bit chunks of E, the exponent of the final 2^res in
    genefer::GL (src/genefer.h:583-592)."""
    bits = np.unpackbits(np.ascontiguousarray(words, dtype="<u4").view(np.uint8), bitorder="little")[:nbits]
    nch = (nbits + B - 1) // B
    padded = np.zeros(nch * B, dtype=np.int64)
    padded[:nbits] = bits
    cs = padded.reshape(nch, B).sum(axis=0)
    res = 0
    for i in range(B - 1, -1, -1):
        res = (res << 1) + int(cs[i])
    return res


def _int_to_words(v: int, nbits: int) -> np.ndarray:
    nw = max(1, (int(nbits) + 31) // 32)
    return np.frombuffer(int(v).to_bytes(4 * nw, "little"), dtype="<u4").astype(np.uint32)


def prefix_words(b: int, n: int, bits: int) -> Tuple[np.ndarray, int, int]:
    """The top ``bits`` bits of E = b^(2^n) without forming E: returns
    (words of the prefix, its bit count, bit length of E).

    E is bracketed by squaring lower and upper bounds truncated to bits + 64
    bits (floor and ceiling); the prefix is exact when both bounds give the
    same bit length and the same top bits, which fails only if E's bits below
    the prefix are all 0 or all 1 for about 64 - n positions.  Then, and for
    prefixes of (nearly) the whole exponent, E is computed in full."""
    b, n, bits = int(b), int(n), int(bits)
    P = bits + 64
    lo = hi = b
    e = 0
    for _ in range(n):
        lo, hi, e = lo * lo, hi * hi, 2 * e
        s = lo.bit_length() - P
        if s > 0:
            lo >>= s
            hi = -((-hi) >> s)
            e += s
    nb_lo, nb_hi = lo.bit_length() + e, hi.bit_length() + e
    if (e > 0) and (nb_lo == nb_hi) and (nb_lo - bits - e >= 0):
        sh = nb_lo - bits - e
        if (lo >> sh) == (hi >> sh):
            return _int_to_words(lo >> sh, bits), bits, nb_lo
    words, nb = exponent_words(b, n)
    if bits >= nb:
        return words, nb, nb
    v = words_to_int(words) >> (nb - bits)
    return _int_to_words(v, bits), bits, nb
