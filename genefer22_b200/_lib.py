"""ctypes binding of libgfcuda.so (include/gfcuda.h).

The library is built in-tree by ``genefer22_b200.build``; importing this
module never falls back to anything else: a missing library raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_lib = None

c_i32p = ctypes.POINTER(ctypes.c_int32)
c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_i64p = ctypes.POINTER(ctypes.c_int64)
vp = ctypes.c_void_p

GFC_OK = 0
ERRORS = {-1: "GFC_ERR_ARG", -2: "GFC_ERR_CUDA", -3: "GFC_ERR_RANGE", -4: "GFC_ERR_NUMERIC", -5: "GFC_ERR_STATE"}

# name: (restype, argtypes); every symbol declared in include/gfcuda.h
SIGNATURES = {
    "gfc_last_error": (ctypes.c_char_p, []),
    "gfc_version": (ctypes.c_int, []),
    "gfc_create": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_size_t, ctypes.c_int, vp, ctypes.POINTER(vp)]),
    "gfc_destroy": (None, [vp]),
    "gfc_set": (ctypes.c_int, [vp, ctypes.c_uint32]),
    "gfc_square_dup": (ctypes.c_int, [vp, ctypes.c_int]),
    "gfc_square_mul": (ctypes.c_int, [vp, ctypes.c_int32]),
    "gfc_init_multiplicand": (ctypes.c_int, [vp, ctypes.c_size_t]),
    "gfc_mul": (ctypes.c_int, [vp]),
    "gfc_copy": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_size_t]),
    "gfc_get_zi": (ctypes.c_int, [vp, c_i32p]),
    "gfc_set_zi": (ctypes.c_int, [vp, c_i32p]),
    "gfc_get_mem_size": (ctypes.c_size_t, [vp]),
    "gfc_get_cache_size": (ctypes.c_size_t, [vp]),
    "gfc_context_size": (ctypes.c_size_t, [vp, ctypes.c_size_t]),
    "gfc_save_context": (ctypes.c_int, [vp, vp, ctypes.c_size_t, ctypes.c_size_t]),
    "gfc_read_context": (ctypes.c_int, [vp, vp, ctypes.c_size_t, ctypes.c_size_t]),
    "gfc_width": (ctypes.c_int, [vp]),
    "gfc_sync": (ctypes.c_int, [vp]),
    "gfc_batch_create": (ctypes.c_int, [c_u32p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_size_t, ctypes.c_int, vp,
                                        ctypes.POINTER(vp)]),
    "gfc_batch_destroy": (None, [vp]),
    "gfc_batch_count": (ctypes.c_size_t, [vp]),
    "gfc_batch_set": (ctypes.c_int, [vp, ctypes.c_uint32]),
    "gfc_batch_copy": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_size_t]),
    "gfc_batch_square": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_uint32]),
    "gfc_batch_set_exponent": (ctypes.c_int, [vp, ctypes.c_size_t, c_u32p, ctypes.c_uint64]),
    "gfc_batch_assign": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_uint32]),
    "gfc_batch_set_pos": (ctypes.c_int, [vp, c_i64p]),
    "gfc_batch_get_pos": (ctypes.c_int, [vp, c_i64p]),
    "gfc_batch_square_exp": (ctypes.c_int, [vp, ctypes.c_uint32]),
    "gfc_batch_init_multiplicand": (ctypes.c_int, [vp, ctypes.c_size_t]),
    "gfc_batch_mul": (ctypes.c_int, [vp, ctypes.c_size_t]),
    "gfc_batch_gl_step": (ctypes.c_int, [vp]),
    "gfc_batch_get_zi": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_size_t, c_i32p]),
    "gfc_batch_set_zi": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_size_t, c_i32p]),
    "gfc_batch_get_all": (ctypes.c_int, [vp, ctypes.c_size_t, c_i32p]),
    "gfc_batch_set_all": (ctypes.c_int, [vp, ctypes.c_size_t, c_i32p]),
    "gfc_batch_set_plan": (ctypes.c_int, [vp, ctypes.c_int]),
    "gfc_batch_plan": (ctypes.c_int, [vp]),
    "gfc_batch_widths": (ctypes.c_int, [vp, c_i32p]),
    "gfc_batch_sync": (ctypes.c_int, [vp]),
    "gfc_batch_time_kernels": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float)]),
    "gfc_batch_stream": (vp, [vp]),
    "gfc_batch_capture_begin": (ctypes.c_int, [vp]),
    "gfc_batch_capture_end": (ctypes.c_int, [vp, ctypes.POINTER(vp)]),
    "gfc_graph_launch": (ctypes.c_int, [vp]),
    "gfc_graph_destroy": (None, [vp]),
    "gfc_launch_count": (ctypes.c_uint64, []),
    "gfc_probe_int_throughput": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "gfc_square_noalloc": (ctypes.c_int, [c_i32p, c_i32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                          ctypes.c_uint32, ctypes.c_int, vp]),
    "gfc_gint_unbalance": (None, [c_i32p, ctypes.c_size_t, ctypes.c_uint32]),
    "gfc_gint_balance": (None, [c_i32p, ctypes.c_size_t, ctypes.c_uint32]),
    "gfc_gint_is_one": (ctypes.c_int, [c_i32p, ctypes.c_size_t, ctypes.c_uint32, c_u64p, c_u64p]),
    "gfc_gint_hash64": (ctypes.c_uint64, [c_i32p, ctypes.c_size_t]),
}


class GfcError(RuntimeError):
    """A libgfcuda call returned a negative status (std::runtime_error in the
    reference's transformGPU, src/ocl.h:166-175)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def lib_path() -> str:
    return _build.LIB


def lib():
    """Loads libgfcuda.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            raise RuntimeError(f"libgfcuda.so not built ({path}); run python -m genefer22_b200.build")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != GFC_OK:
        raise GfcError(code, lib().gfc_last_error().decode(errors="replace"))
