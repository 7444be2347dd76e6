"""genefer's ``gint`` residue utilities (src/gint.h:40-225) on numpy digit
vectors, computed by libgfcuda's host functions."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import c_i32p, lib


def _arr(d) -> np.ndarray:
    return np.array(d, dtype=np.int32, copy=True, order="C")


def unbalance(d, b: int) -> np.ndarray:
    """Canonical digits in [0, b) (gint::unbalance, src/gint.h:40-102)."""
    x = _arr(d)
    lib().gfc_gint_unbalance(x.ctypes.data_as(c_i32p), x.size, b)
    return x


def balance(d, b: int) -> np.ndarray:
    """Digits in (-b/2, b/2] (gint::balance, src/gint.h:104-149)."""
    x = _arr(d)
    lib().gfc_gint_balance(x.ctypes.data_as(c_i32p), x.size, b)
    return x


def is_one(canon: np.ndarray, b: int):
    """(isOne, res64, old64) of canonical digits (gint::isOne, src/gint.h:169-202)."""
    x = np.ascontiguousarray(canon, dtype=np.int32)
    r, o = ctypes.c_uint64(0), ctypes.c_uint64(0)
    one = lib().gfc_gint_is_one(x.ctypes.data_as(c_i32p), x.size, b, ctypes.byref(r), ctypes.byref(o))
    return bool(one), int(r.value), int(o.value)


def hash64(canon: np.ndarray) -> int:
    """gint::gethash64 of canonical digits (src/gint.h:204-219)."""
    x = np.ascontiguousarray(canon, dtype=np.int32)
    return int(lib().gfc_gint_hash64(x.ctypes.data_as(c_i32p), x.size))


def res64(d, b: int) -> int:
    return is_one(unbalance(d, b), b)[1]
