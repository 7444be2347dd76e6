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

class ServerConfig(ctypes.Structure):
    """gfc_server_config (include/gfcuda.h)."""
    _fields_ = [("block", ctypes.c_uint32), ("validate_group", ctypes.c_uint32), ("budget_bytes", ctypes.c_uint64),
                ("capacity", ctypes.c_uint32 * 24), ("device", ctypes.c_int32), ("tune", ctypes.c_int32),
                ("keep_digits", ctypes.c_int32), ("idle_close_s", ctypes.c_double)]


class CompletionC(ctypes.Structure):
    """gfc_completion (include/gfcuda.h)."""
    _fields_ = [("id", ctypes.c_uint64), ("nbits", ctypes.c_uint64), ("b", ctypes.c_uint32), ("n", ctypes.c_uint32),
                ("arrival", ctypes.c_double), ("admitted", ctypes.c_double), ("residue_at", ctypes.c_double),
                ("validated_at", ctypes.c_double), ("res64", ctypes.c_uint64), ("old64", ctypes.c_uint64),
                ("is_prp", ctypes.c_int32), ("gl_ok", ctypes.c_int32), ("pool", ctypes.c_int32),
                ("slot", ctypes.c_int32), ("plan", ctypes.c_int32)]


class ServerStatsC(ctypes.Structure):
    """gfc_server_stats (include/gfcuda.h)."""
    _fields_ = [(k, ctypes.c_uint64) for k in ("submitted", "completed", "pools_created", "pools_open", "blocks_run",
                                               "used_bytes", "peak_bytes", "budget_bytes", "gl_failures")] + \
        [(k, ctypes.c_double) for k in ("open_s_sum", "open_s_max", "step_s_max")] + [("phase_s_max", ctypes.c_double * 9)]


# The serving loop's entry points (also exported by the CPU build of the same
# loop that the host-logic tests load).
SERVER_SIGNATURES = {
    "gfc_server_default_config": (None, [ctypes.POINTER(ServerConfig)]),
    "gfc_server_create": (ctypes.c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
    "gfc_server_pretune": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.c_uint32]),
    "gfc_server_submit": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, c_u32p, ctypes.c_uint64]),
    "gfc_server_poll": (ctypes.c_int, [vp, ctypes.POINTER(CompletionC), ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_size_t), ctypes.c_int32]),
    "gfc_server_digits": (ctypes.c_int, [vp, ctypes.c_uint64, c_i32p, ctypes.c_size_t]),
    "gfc_server_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServerStatsC)]),
    "gfc_server_clock": (ctypes.c_double, [vp]),
    "gfc_server_destroy": (None, [vp]),
    "gfc_server_slot_bytes": (ctypes.c_uint64, [ctypes.c_uint32, ctypes.c_uint64]),
    "gfc_server_table_bytes": (ctypes.c_uint64, [ctypes.c_uint32]),
    "gfc_server_default_capacity": (ctypes.c_uint32, [ctypes.c_uint32]),
}

# name: (restype, argtypes); every symbol declared in include/gfcuda.h
SIGNATURES = {
    **SERVER_SIGNATURES,
    "gfc_batch_reserve": (ctypes.c_int, [vp, ctypes.c_uint64]),
    "gfc_batch_admit": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_uint32, c_u32p, ctypes.c_uint64]),
    "gfc_batch_get_async": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_size_t, c_i32p]),
    "gfc_batch_set_async": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.c_size_t, c_i32p]),
    "gfc_plan_candidates": (ctypes.c_int, [ctypes.c_uint32, c_i32p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "gfc_batch_tune": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.c_uint32, c_i32p, ctypes.POINTER(ctypes.c_float),
                                      ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), c_i32p]),
    "gfc_width_for": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32]),
    "gfc_packed_range": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32]),
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
