"""gfc_square_noalloc: the squaring entry point for callers that cannot
allocate device memory when they square (it keeps its scratch in a static
device array).  Its output must equal the regular engine's, on two calls in a
row.  This file is collected last so that a failure here leaves every other
test already run."""
import ctypes

import numpy as np
import pytest

from genefer22_b200 import Transform, gint
from genefer22_b200._lib import GFC_OK, c_i32p, lib

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), c_i32p)


@pytest.mark.parametrize("b,n", [(50_000_002, 16), (1_000_002, 12), (1_999_999_998, 14)])
def test_square_noalloc_matches_engine(b, n):
    import torch
    rng = np.random.default_rng(n)
    x = gint.balance(rng.integers(-(b // 2), b // 2 + 1, size=1 << n).astype(np.int32), b)
    t = Transform(b, n)
    t.setInt(x)
    cur = torch.tensor(x, dtype=torch.int32, device="cuda:0")
    out = torch.empty_like(cur)
    torch.cuda.synchronize()
    for call, (dup, count) in enumerate(((1, 3), (0, 2))):
        rc = lib().gfc_square_noalloc(_ptr(cur), _ptr(out), b, n, dup, count, 0, None)
        assert rc == GFC_OK, lib().gfc_last_error().decode()
        for _ in range(count):
            t.squareDup(bool(dup))
        got = out.cpu().numpy()
        assert np.abs(got).max() <= b // 2 + 1
        assert np.array_equal(gint.unbalance(got, b), gint.unbalance(t.getInt(), b)), f"call {call}"
        cur, out = out, cur


def test_square_noalloc_in_place_and_limits():
    import torch
    b, n = 1_000_002, 13
    rng = np.random.default_rng(5)
    x = gint.balance(rng.integers(-(b // 2), b // 2 + 1, size=1 << n).astype(np.int32), b)
    t = Transform(b, n)
    t.setInt(x)
    buf = torch.tensor(x, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    for _ in range(2):
        assert lib().gfc_square_noalloc(_ptr(buf), _ptr(buf), b, n, 0, 1, 0, None) == GFC_OK
        t.squareDup(False)
        assert np.array_equal(gint.unbalance(buf.cpu().numpy(), b), gint.unbalance(t.getInt(), b))
    big = torch.zeros(1 << 17, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    assert lib().gfc_square_noalloc(_ptr(big), _ptr(big), b, 17, 0, 1, 0, None) == -1
    assert b"12 <= n <= 16" in lib().gfc_last_error()


def test_square_noalloc_allocates_nothing():
    """The point of the entry point: once a device is set up, calls take no device memory,
    also when a change of n rebuilds the root tables inside the static array.  The warm-up
    calls load every kernel the later calls launch, so lazy module loading cannot show up
    as an allocation."""
    import torch
    cases = [(1_000_002, 12), (50_000_002, 16)]
    bufs = [torch.zeros(1 << n, dtype=torch.int32, device="cuda:0") for _, n in cases]
    torch.cuda.synchronize()
    for (b, n), buf in zip(cases, bufs):
        assert lib().gfc_square_noalloc(_ptr(buf), _ptr(buf), b, n, 0, 1, 0, None) == GFC_OK
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(2):
        for (b, n), buf in zip(cases, bufs):
            rc = lib().gfc_square_noalloc(_ptr(buf), _ptr(buf), b, n, 1, 2, 0, None)
            assert rc == GFC_OK, lib().gfc_last_error().decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] >= free0


def test_square_noalloc_rejects_partial_overlap():
    import torch
    b, n = 1_000_002, 12
    buf = torch.zeros(2 << n, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    base = buf.data_ptr()
    half = ctypes.cast(ctypes.c_void_p(base + 4 * (1 << (n - 1))), c_i32p)
    assert lib().gfc_square_noalloc(_ptr(buf), half, b, n, 0, 1, 0, None) == -1
    assert b"equal or disjoint" in lib().gfc_last_error()
    far = ctypes.cast(ctypes.c_void_p(base + 4 * (1 << n)), c_i32p)
    assert lib().gfc_square_noalloc(_ptr(buf), far, b, n, 0, 1, 0, None) == GFC_OK
