"""CPU ORACLE wrappers -- test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module, and only as the checker.  It loads

* ``oracle/_build/libgforacle.so`` -- the C restatement of genefer's
  bit-exact integer transform (``transformCPUi32``, src/transformCPUi32.h) and
  of ``gint`` (src/gint.h), built from ``oracle/gf_oracle.c``;
* ``oracle/_ref/libgfref.so`` -- the reference's own CPU transforms compiled
  from the reference sources by ``oracle/Makefile`` (optional; present in the
  build container and carried to GPU runs as a prebuilt file).

It also restates the test driver ``genefer::prp`` / ``genefer::GL`` /
``genefer::quick`` (src/genefer.h:467-615, :736-748) over any object with the
``transform`` API, so KATs from the reference sources can be checked.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "_build", "libgforacle.so")
REF_SO = os.path.join(_HERE, "_ref", "libgfref.so")

_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)

_lib = None
_ref = None


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle)")
        L = ctypes.CDLL(ORACLE_SO)
        L.gfo_create.restype = ctypes.c_void_p
        L.gfo_create.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_size_t]
        L.gfo_destroy.argtypes = [ctypes.c_void_p]
        L.gfo_set.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.gfo_square_dup.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.gfo_square_mul.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.gfo_init_multiplicand.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        L.gfo_mul.argtypes = [ctypes.c_void_p]
        L.gfo_copy.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t]
        L.gfo_get_zi.argtypes = [ctypes.c_void_p, _i32p]
        L.gfo_set_zi.argtypes = [ctypes.c_void_p, _i32p]
        L.gfo_get_raw.argtypes = [ctypes.c_void_p, _u32p]
        L.gfo_unbalance.argtypes = [_i32p, ctypes.c_size_t, ctypes.c_uint32]
        L.gfo_balance.argtypes = [_i32p, ctypes.c_size_t, ctypes.c_uint32]
        L.gfo_is_one.restype = ctypes.c_int
        L.gfo_is_one.argtypes = [_i32p, ctypes.c_size_t, ctypes.c_uint32, _u64p, _u64p]
        L.gfo_hash64.restype = ctypes.c_uint64
        L.gfo_hash64.argtypes = [_i32p, ctypes.c_size_t]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"reference library missing: {REF_SO} (run make -C oracle ref)")
        L = ctypes.CDLL(REF_SO)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_create.restype = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_size_t, ctypes.c_char_p,
                                 ctypes.c_size_t, ctypes.c_int]
        L.ref_type.restype = ctypes.c_char_p
        L.ref_type.argtypes = [ctypes.c_void_p]
        L.ref_destroy.argtypes = [ctypes.c_void_p]
        L.ref_set.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.ref_square_dup.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_square_mul.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.ref_init_multiplicand.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        L.ref_mul.argtypes = [ctypes.c_void_p]
        L.ref_copy.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t]
        L.ref_get_error.restype = ctypes.c_double
        L.ref_get_error.argtypes = [ctypes.c_void_p]
        L.ref_run_squarings.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_size_t]
        L.ref_get_zi.argtypes = [ctypes.c_void_p, _i32p]
        L.ref_set_zi.argtypes = [ctypes.c_void_p, _i32p]
        L.ref_save_raw.restype = ctypes.c_long
        L.ref_save_raw.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
        _ref = L
    return _ref


# ---------------------------------------------------------------- gint

def unbalance(d: np.ndarray, b: int) -> np.ndarray:
    """gint::unbalance (src/gint.h:40-102): canonical digits in [0, b)."""
    x = np.ascontiguousarray(d, dtype=np.int32).copy()
    lib().gfo_unbalance(_ptr(x, _i32p), x.size, b)
    return x


def balance(d: np.ndarray, b: int) -> np.ndarray:
    """gint::balance (src/gint.h:104-149): digits in (-b/2, b/2]."""
    x = np.ascontiguousarray(d, dtype=np.int32).copy()
    lib().gfo_balance(_ptr(x, _i32p), x.size, b)
    return x


def is_one(d_unbalanced: np.ndarray, b: int):
    """gint::isOne (src/gint.h:169-202) on canonical digits: (isOne, res64, old64)."""
    x = np.ascontiguousarray(d_unbalanced, dtype=np.int32)
    r = ctypes.c_uint64(0)
    o = ctypes.c_uint64(0)
    one = lib().gfo_is_one(_ptr(x, _i32p), x.size, b, ctypes.byref(r), ctypes.byref(o))
    return bool(one), r.value, o.value


def hash64(d_unbalanced: np.ndarray) -> int:
    """gint::gethash64 (src/gint.h:204-219) on canonical digits."""
    x = np.ascontiguousarray(d_unbalanced, dtype=np.int32)
    return int(lib().gfo_hash64(_ptr(x, _i32p), x.size))


# ---------------------------------------------------------------- transforms

class OracleTransform:
    """The C restatement of transformCPUi32 behind the reference's transform API."""

    def __init__(self, b: int, n: int, num_regs: int = 3):
        self.b, self.n, self.size = b, n, 1 << n
        self._h = lib().gfo_create(b, n, num_regs)
        if not self._h:
            raise RuntimeError(f"gfo_create({b}, {n}) failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().gfo_destroy(h)
            self._h = None

    def set(self, a: int):
        lib().gfo_set(self._h, a)

    def squareDup(self, dup: bool):
        lib().gfo_square_dup(self._h, 1 if dup else 0)

    def squareMul(self, a: int):
        lib().gfo_square_mul(self._h, a)

    def initMultiplicand(self, src: int):
        lib().gfo_init_multiplicand(self._h, src)

    def mul(self, src: Optional[int] = None):
        if src is not None:
            self.initMultiplicand(src)
        lib().gfo_mul(self._h)

    def copy(self, dst: int, src: int):
        lib().gfo_copy(self._h, dst, src)

    def getInt(self) -> np.ndarray:
        out = np.empty(self.size, dtype=np.int32)
        lib().gfo_get_zi(self._h, _ptr(out, _i32p))
        return out

    def setInt(self, d: np.ndarray):
        x = balance(d, self.b)
        lib().gfo_set_zi(self._h, _ptr(x, _i32p))

    def raw(self) -> np.ndarray:
        out = np.empty(3 * self.size, dtype=np.uint32)
        lib().gfo_get_raw(self._h, _ptr(out, _u32p))
        return out


class RefTransform:
    """The reference's own CPU transform (oracle/_ref), via transform::create_cpu."""

    def __init__(self, b: int, n: int, num_regs: int = 3, impl: str = "i32", threads: int = 1,
                 check_error: bool = False):
        L = ref_lib()
        self.b, self.n, self.size = b, n, 1 << n
        self._h = L.ref_create(b, n, num_regs, impl.encode(), threads, 1 if check_error else 0)
        if not self._h:
            raise RuntimeError(f"ref_create failed: {L.ref_last_error().decode()}")
        self.ttype = L.ref_type(self._h).decode()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            ref_lib().ref_destroy(h)
            self._h = None

    def set(self, a: int):
        ref_lib().ref_set(self._h, a)

    def squareDup(self, dup: bool):
        ref_lib().ref_square_dup(self._h, 1 if dup else 0)

    def squareMul(self, a: int):
        ref_lib().ref_square_mul(self._h, a)

    def run_squarings(self, bits: np.ndarray):
        x = np.ascontiguousarray(bits, dtype=np.uint8)
        ref_lib().ref_run_squarings(self._h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), x.size)

    def initMultiplicand(self, src: int):
        ref_lib().ref_init_multiplicand(self._h, src)

    def mul(self, src: Optional[int] = None):
        if src is not None:
            self.initMultiplicand(src)
        ref_lib().ref_mul(self._h)

    def copy(self, dst: int, src: int):
        ref_lib().ref_copy(self._h, dst, src)

    def getInt(self) -> np.ndarray:
        out = np.empty(self.size, dtype=np.int32)
        ref_lib().ref_get_zi(self._h, _ptr(out, _i32p))
        return out

    def setInt(self, d: np.ndarray):
        x = np.ascontiguousarray(d, dtype=np.int32)
        ref_lib().ref_set_zi(self._h, _ptr(x, _i32p))

    def raw(self) -> np.ndarray:
        """Register 0 as [N/4][3 primes][4 lanes] uint32, like OracleTransform.raw().

        The reference stores each prime's 4 lanes in the even 32-bit slots of
        a 256-bit vector (src/transformCPUi32.h:115-131)."""
        buf = np.empty(6 * self.size, dtype=np.uint32)
        got = ref_lib().ref_save_raw(self._h, buf.ctypes.data, buf.nbytes)
        if got != buf.nbytes:
            raise RuntimeError("ref_save_raw failed")
        return buf.reshape(self.size // 4, 3, 8)[:, :, 0::2].reshape(-1).copy()


# ---------------------------------------------------------------- driver

def exponent(b: int, n: int) -> int:
    """E = b^(2^n) (src/genefer.h:1476)."""
    return b ** (1 << n)


def B_GerbiczLi(esize: int) -> int:
    """genefer::B_GerbiczLi (src/genefer.h:467-471)."""
    L = 2 << ((esize.bit_length() - 1) // 2)
    return (esize - 1) // L + 1


def prp(t, E: int, B_GL: int):
    """genefer::prp without checkpoints/proof (src/genefer.h:479-552):
    out reg0 = 2^E, reg1 = d(t)."""
    t.set(1)
    t.copy(1, 0)
    for i in range(E.bit_length() - 1, -1, -1):
        t.squareDup(((E >> i) & 1) != 0)
        if (i % B_GL == 0) and (i // B_GL != 0):
            t.copy(2, 0)
            t.mul(1)
            t.copy(1, 0)
            t.copy(0, 2)


def GL(t, E: int, B_GL: int, b: int) -> bool:
    """genefer::GL (src/genefer.h:557-615)."""
    t.mul(1)
    t.copy(2, 0)
    t.copy(0, 1)
    for _ in range(B_GL):
        t.squareDup(False)
    t.copy(1, 0)
    res, e = 0, E
    mask = (1 << B_GL) - 1
    while e:
        res += e & mask
        e >>= B_GL
    t.set(1)
    for i in range(res.bit_length() - 1, -1, -1):
        t.squareDup(((res >> i) & 1) != 0)
    t.mul(1)
    h1 = hash64(unbalance(t.getInt(), b))
    t.copy(0, 2)
    h2 = hash64(unbalance(t.getInt(), b))
    return h1 == h2


def quick(t, b: int, n: int, E: Optional[int] = None):
    """genefer::quick (src/genefer.h:736-748): returns (isPrp, res64, old64, gl_ok)."""
    if E is None:
        E = exponent(b, n)
    B = B_GerbiczLi(E.bit_length())
    prp(t, E, B)
    is_prp, res64, old64 = is_one(unbalance(t.getInt(), b), b)
    ok = GL(t, E, B, b)
    return is_prp, res64, old64, ok
