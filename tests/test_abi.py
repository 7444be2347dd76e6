"""CPU tests of the product's host side: the C ABI loads and exports every
declared symbol, and the host-only functions (gint, exponent, schedule)
agree with the oracle.  No GPU work is launched here."""
import os
import re

import numpy as np
import pytest

from genefer22_b200 import _lib, gint
from genefer22_b200 import exponent as ex

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gfcuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gfc_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header():
    L = _lib.lib()
    syms = declared_symbols()
    assert len(syms) > 30
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES), set(syms) ^ set(_lib.SIGNATURES)


def test_version():
    assert _lib.lib().gfc_version() == 100


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from genefer22_b200 import Transform, GfcError
    with pytest.raises(GfcError):
        Transform(1000, 12)


def test_batch_arguments_checked_before_device_work():
    """Out-of-range batch arguments fail with GFC_ERR_ARG before any CUDA
    call, so this runs without a GPU."""
    from genefer22_b200 import GfcError
    from genefer22_b200.transform import Batch
    for bases, n, regs in (([1000] * 65536, 12, 3), ([1000], 9, 3), ([1000], 24, 3), ([1000], 12, 0)):
        with pytest.raises(GfcError) as e:
            Batch(bases, n, regs)
        assert e.value.code == -1, e.value


def test_gint_matches_oracle(oracle):
    rng = np.random.default_rng(3)
    for b in (1024, 65538, 2 * 10**9 - 2):
        d = rng.integers(-(b // 2) - 1, b // 2 + 2, size=4096).astype(np.int32)
        assert np.array_equal(gint.unbalance(d, b), oracle.unbalance(d, b))
        assert np.array_equal(gint.balance(d, b), oracle.balance(d, b))
        c = oracle.unbalance(d, b)
        assert gint.is_one(c, b) == oracle.is_one(c, b)
        assert gint.hash64(c) == oracle.hash64(c)


def test_gint_minus_one_and_one(oracle):
    b, N = 1000, 64
    d = np.zeros(N, np.int32)
    d[0] = -1
    assert np.array_equal(gint.unbalance(d, b), oracle.unbalance(d, b))
    d[0] = 1
    assert gint.is_one(gint.unbalance(d, b), b)[0]


@pytest.mark.parametrize("b,n", [(1024, 5), (10**9, 8), (2 * 10**9 - 2, 10), (12345678, 12)])
def test_exponent_words(b, n):
    w, nb = ex.exponent_words(b, n)
    E = pow(b, 1 << n)
    assert nb == E.bit_length()
    assert ex.words_to_int(w) == E


def test_b_gl_and_chunk_sum(oracle):
    for b, n in ((10**6, 12), (5 * 10**7, 16)):
        w, nb = ex.exponent_words(b, n)
        B = ex.B_GerbiczLi(nb)
        assert B == oracle.B_GerbiczLi(nb)
        E, res, e = ex.words_to_int(w), 0, None
        e = E
        while e:
            res += e & ((1 << B) - 1)
            e >>= B
        assert ex.chunk_sum(w, nb, B) == res


def test_survey_b_gl_values():
    # |E| = 81,640 (n=12, b=10^6) gives B_GL = 160 (src/genefer.h:467-471)
    assert ex.B_GerbiczLi(81640) == 160
