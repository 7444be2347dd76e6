"""Python mirror of genefer's ``transform`` interface over libgfcuda.

``Transform`` follows src/transform.h:42-256 (same member names and meaning:
set / squareDup / initMultiplicand / mul / copy / getInt / setInt /
getMemSize / getCacheSize / saveContext / readContext); errors raise
``GfcError`` as the reference raises std::runtime_error.  ``Batch`` is the
many-tests-per-launch extension and ``Graph`` a captured CUDA graph.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from ._lib import GfcError, c_i32p, c_i64p, c_u32p, check, lib
from . import gint


def _i32(a: np.ndarray):
    return a.ctypes.data_as(c_i32p)


class Batch:
    """count tests of one size n (each with its own base b) on one device."""

    def __init__(self, bases: Sequence[int], n: int, num_regs: int = 3, device: int = 0, stream: Optional[int] = None):
        L = lib()
        self.bases = np.ascontiguousarray(np.asarray(bases, dtype=np.uint32))
        self.n, self.size, self.count, self.num_regs = int(n), 1 << int(n), int(self.bases.size), int(num_regs)
        h = ctypes.c_void_p()
        check(L.gfc_batch_create(self.bases.ctypes.data_as(c_u32p), self.count, self.n, self.num_regs, device,
                                 ctypes.c_void_p(stream) if stream else None, ctypes.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self._h = None
            try:
                lib().gfc_batch_destroy(h)
            except Exception:   # interpreter shutdown
                pass

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return int(lib().gfc_batch_stream(self._h) or 0)

    def widths(self) -> np.ndarray:
        w = np.empty(self.count, dtype=np.int32)
        check(lib().gfc_batch_widths(self._h, _i32(w)))
        return w

    def plan(self) -> int:
        return int(lib().gfc_batch_plan(self._h))

    def set_plan(self, lr: int):
        check(lib().gfc_batch_set_plan(self._h, int(lr)))

    def set(self, a: int):
        check(lib().gfc_batch_set(self._h, a))

    def copy(self, dst: int, src: int):
        check(lib().gfc_batch_copy(self._h, dst, src))

    def square(self, dup: bool = False, count: int = 1):
        check(lib().gfc_batch_square(self._h, 1 if dup else 0, count))

    def set_exponent(self, test: int, words: np.ndarray, nbits: int):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        check(lib().gfc_batch_set_exponent(self._h, test, w.ctypes.data_as(c_u32p), nbits))

    def assign(self, test: int, b: int):
        """Slot `test` now holds a test of base b (registers unchanged)."""
        check(lib().gfc_batch_assign(self._h, test, b))
        self.bases[test] = b

    def reserve(self, max_bits: int):
        """Room for exponents of up to max_bits bits in every slot, once, so that
        ``admit`` allocates nothing and never synchronises (gfc_batch_reserve)."""
        check(lib().gfc_batch_reserve(self._h, int(max_bits)))

    def admit(self, test: int, b: int, words: np.ndarray, nbits: int):
        """A new test in slot ``test``: base b, r0 = r1 = 1, exponent, position;
        enqueued on the batch stream (gfc_batch_admit)."""
        w = np.ascontiguousarray(words, dtype=np.uint32)
        check(lib().gfc_batch_admit(self._h, test, int(b), w.ctypes.data_as(c_u32p), int(nbits)))
        self.bases[test] = b

    def set_pos(self, pos: Sequence[int]):
        p = np.ascontiguousarray(np.asarray(pos, dtype=np.int64))
        check(lib().gfc_batch_set_pos(self._h, p.ctypes.data_as(c_i64p)))

    def get_pos(self) -> np.ndarray:
        p = np.empty(self.count, dtype=np.int64)
        check(lib().gfc_batch_get_pos(self._h, p.ctypes.data_as(c_i64p)))
        return p

    def square_exp(self, count: int):
        check(lib().gfc_batch_square_exp(self._h, count))

    def init_multiplicand(self, src: int):
        check(lib().gfc_batch_init_multiplicand(self._h, src))

    def mul_into(self, dst: int):
        check(lib().gfc_batch_mul(self._h, dst))

    def gl_step(self):
        check(lib().gfc_batch_gl_step(self._h))

    def get(self, test: int, reg: int = 0) -> np.ndarray:
        out = np.empty(self.size, dtype=np.int32)
        check(lib().gfc_batch_get_zi(self._h, test, reg, _i32(out)))
        return out

    def put(self, test: int, digits: np.ndarray, reg: int = 0):
        x = np.ascontiguousarray(digits, dtype=np.int32)
        check(lib().gfc_batch_set_zi(self._h, test, reg, _i32(x)))

    def get_all(self, reg: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.count, self.size), dtype=np.int32)
        check(lib().gfc_batch_get_all(self._h, reg, _i32(out)))
        return out

    def put_all(self, digits: np.ndarray, reg: int = 0):
        x = np.ascontiguousarray(digits, dtype=np.int32)
        check(lib().gfc_batch_set_all(self._h, reg, _i32(x)))

    def sync(self):
        check(lib().gfc_batch_sync(self._h))

    def time_kernels(self, reps: int = 5) -> np.ndarray:
        """Mean ms per squaring of each kernel kind: [single-CTA, column-forward,
        row, column-inverse + carry, carry fix-up]."""
        ms = (ctypes.c_float * 5)()
        check(lib().gfc_batch_time_kernels(self._h, reps, ms))
        return np.array(list(ms), dtype=np.float64)

    def capture(self, fn) -> "Graph":
        """Records the batch calls made by fn() into a CUDA graph."""
        check(lib().gfc_batch_capture_begin(self._h))
        g = ctypes.c_void_p()
        try:
            fn()
        finally:
            rc = lib().gfc_batch_capture_end(self._h, ctypes.byref(g))
        check(rc)
        return Graph(g)


class Graph:
    def __init__(self, h):
        self._h = h

    def launch(self):
        check(lib().gfc_graph_launch(self._h))

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self._h = None
            try:
                lib().gfc_graph_destroy(h)
            except Exception:   # interpreter shutdown
                pass

    __del__ = close


class Transform:
    """One test behind genefer's transform API (src/transform.h:42-256)."""

    def __init__(self, b: int, n: int, num_regs: int = 3, device: int = 0, stream: Optional[int] = None):
        self._batch = Batch([b], n, num_regs, device, stream)
        self.b, self.n, self.size = int(b), int(n), 1 << int(n)

    # transform::set / squareDup / initMultiplicand / mul / copy (src/transform.h:58-64)
    def set(self, a: int):
        check(lib().gfc_set(self._batch.handle, a))

    def squareDup(self, dup: bool):
        check(lib().gfc_square_dup(self._batch.handle, 1 if dup else 0))

    def squareMul(self, a: int):
        """r_0 = a r_0^2 (transform::squareMul, src/transform.h:60)."""
        check(lib().gfc_square_mul(self._batch.handle, a))

    def initMultiplicand(self, src: int):
        check(lib().gfc_init_multiplicand(self._batch.handle, src))

    def mul(self, src: Optional[int] = None):
        """mul() or, with src, the non-virtual mul(src) (src/transform.h:228-232)."""
        if src is not None:
            self.initMultiplicand(src)
        check(lib().gfc_mul(self._batch.handle))

    def copy(self, dst: int, src: int):
        check(lib().gfc_copy(self._batch.handle, dst, src))

    # transform::getInt / setInt (src/transform.h:234-246)
    def getInt(self) -> np.ndarray:
        out = np.empty(self.size, dtype=np.int32)
        check(lib().gfc_get_zi(self._batch.handle, _i32(out)))
        return out

    def setInt(self, digits: np.ndarray):
        x = gint.balance(digits, self.b)
        check(lib().gfc_set_zi(self._batch.handle, _i32(x)))

    def getMemSize(self) -> int:
        return int(lib().gfc_get_mem_size(self._batch.handle))

    def getCacheSize(self) -> int:
        return int(lib().gfc_get_cache_size(self._batch.handle))

    def contextSize(self, num_regs: int) -> int:
        """Bytes of saveContext(num_regs); num_regs 0 means every register, as
        in the reference's readContext / saveContext (src/transformGPU.h:1127-1150)."""
        return int(lib().gfc_context_size(self._batch.handle, num_regs or self._batch.num_regs))

    def saveContext(self, num_regs: int) -> bytes:
        num_regs = num_regs or self._batch.num_regs
        size = int(lib().gfc_context_size(self._batch.handle, num_regs))
        buf = ctypes.create_string_buffer(size)
        check(lib().gfc_save_context(self._batch.handle, buf, size, num_regs))
        return buf.raw

    def readContext(self, data: bytes, num_regs: int) -> bool:
        num_regs = num_regs or self._batch.num_regs
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        rc = lib().gfc_read_context(self._batch.handle, buf, len(data), num_regs)
        if rc == -5:
            return False
        check(rc)
        return True

    def width(self) -> int:
        return int(lib().gfc_width(self._batch.handle))

    def sync(self):
        check(lib().gfc_sync(self._batch.handle))

    @property
    def batch(self) -> Batch:
        return self._batch


__all__ = ["Batch", "Graph", "Transform", "GfcError"]
