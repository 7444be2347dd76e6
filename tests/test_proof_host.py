"""genefer's file formats and the proof / server / check protocol, on the CPU.

The protocol runs over the oracle transform (restated transformCPUi32) at a
small size; the GPU tests run the same module over the CUDA engine."""
import ctypes
import ctypes.util
import os

import numpy as np
import pytest

from genefer22_b200 import gint
from genefer22_b200 import proof as pf
from genefer22_b200.exponent import _load_gmp


def test_crc_roundtrip(tmp_path):
    p = str(tmp_path / "x.bin")
    with pf.GFile(p, "wb") as f:
        f.write_i32(-1)
        f.write_f64(2.5)
        f.write(b"genefer")
        f.write_mpz(123456789 ** 5)
        f.write_crc32()
    with pf.GFile(p, "rb") as f:
        assert f.read_i32() == -1 and f.read_f64() == 2.5 and f.read(7) == b"genefer"
        assert f.read_mpz() == 123456789 ** 5
        assert f.check_crc32()
    raw = bytearray(open(p, "rb").read())
    raw[5] ^= 1
    open(p, "wb").write(bytes(raw))
    with pf.GFile(p, "rb") as f:
        f.read_i32(); f.read_f64(); f.read(7); f.read_mpz()
        assert not f.check_crc32()


def test_crc_is_standard_crc32():
    # the table of src/file.h:71-104 is the reflected 0xEDB88320 CRC-32
    import zlib
    assert zlib.crc32(b"123456789") == 0xCBF43926


@pytest.mark.parametrize("v", [0, 1, 255, 256, 2 ** 64 + 3, -(2 ** 70) - 1, 7 ** 300])
def test_mpz_raw_matches_gmp(tmp_path, v):
    """write_mpz / read_mpz against GMP's own mpz_out_raw / mpz_inp_raw."""
    g = _load_gmp()
    if g is None:
        pytest.skip("libgmp not present")
    libc = ctypes.CDLL(ctypes.util.find_library("c"))
    libc.fopen.restype = ctypes.c_void_p
    libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    libc.fclose.argtypes = [ctypes.c_void_p]
    g.__gmpz_out_raw.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    g.__gmpz_inp_raw.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    g.__gmpz_set_str.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
    g.__gmpz_get_str.restype = ctypes.c_void_p
    g.__gmpz_get_str.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p]
    z = ctypes.create_string_buffer(32)
    g.__gmpz_init(z)
    try:
        g.__gmpz_set_str(z, str(v).encode(), 10)
        p_gmp = str(tmp_path / "gmp.raw").encode()
        fp = libc.fopen(p_gmp, b"wb")
        g.__gmpz_out_raw(fp, z)
        libc.fclose(fp)
        p_ours = str(tmp_path / "ours.raw")
        with pf.GFile(p_ours, "wb") as f:
            f.write_mpz(v)
        assert open(p_gmp, "rb").read() == open(p_ours, "rb").read()
        g.__gmpz_set_str(z, b"0", 10)
        fp = libc.fopen(p_ours.encode(), b"rb")
        g.__gmpz_inp_raw(z, fp)
        libc.fclose(fp)
        s = ctypes.create_string_buffer(4096)
        g.__gmpz_get_str(s, 10, z)
        assert int(s.value.decode()) == v
    finally:
        g.__gmpz_clear(z)


def test_gint_format(tmp_path):
    rng = np.random.default_rng(1)
    b, N = 1_000_002, 1024
    d = rng.integers(-(b // 2), b // 2 + 1, size=N).astype(np.int32)
    p = str(tmp_path / "g.bin")
    with pf.GFile(p, "wb") as f:
        pf.write_gint(f, d, b)
    raw = open(p, "rb").read()
    assert len(raw) == 8 + 4 * N
    assert np.frombuffer(raw[:8], "<u4").tolist() == [N, b]
    with pf.GFile(p, "rb") as f:
        assert np.array_equal(pf.read_gint(f, N, b), gint.unbalance(d, b))
    with pf.GFile(p, "rb") as f:
        with pytest.raises(pf.FileError):
            pf.read_gint(f, N, b + 2)


class _CtxOnly:
    """A transform stand-in holding two registers as bytes."""

    def __init__(self, payload=b"\x01" * 16):
        self.payload = payload

    def contextSize(self, num_regs):
        return 16

    def saveContext(self, num_regs):
        return self.payload

    def readContext(self, data, num_regs):
        self.payload = data
        return True


def test_context_files(tmp_path):
    p = str(tmp_path / "t.ctx")
    t = _CtxOnly(b"A" * 16)
    pf.save_context(p, t, 0, 1234, 5.5, 2)
    t.payload = b"B" * 16
    pf.save_context(p, t, 0, 1000, 6.5, 2)
    assert os.path.exists(p) and os.path.exists(p + ".old") and not os.path.exists(p + ".new")
    u = _CtxOnly(b"?" * 16)
    assert pf.read_context(p, u, 0, 2) == (1000, 6.5) and u.payload == b"B" * 16
    assert pf.read_context(p, u, 1, 2) is None                  # other mode
    raw = bytearray(open(p, "rb").read())
    raw[20] ^= 4                                                # damaged: falls back to .old
    open(p, "wb").write(bytes(raw))
    assert pf.read_context(p, u, 0, 2) == (1234, 5.5) and u.payload == b"A" * 16


def _oracle_chain(oracle, tmp_path, b, n, depth, rnd):
    t = oracle.OracleTransform(b, n, 3 + (1 << depth))
    pr = pf.proof(t, b, n, depth, str(tmp_path / "p.proof"))
    s = pf.server(oracle.OracleTransform(b, n, 4), b, n, str(tmp_path / "p.proof"), str(tmp_path / "p.cert"), rnd)
    ck = pf.check(oracle.OracleTransform(b, n, 4), b, n, str(tmp_path / "p.cert"))
    return pr, s, ck


def test_proof_server_check_on_oracle(oracle, tmp_path):
    """The client's pkey is the server's, the checker's ckey is the server's,
    and the proof's first residue is the test's."""
    b, n = 1_000_002, 10
    pr, s, ck = _oracle_chain(oracle, tmp_path, b, n, 3, (17, 100, 3000))
    o = oracle.OracleTransform(b, n)
    isp, r64, o64, ok = oracle.quick(o, b, n)
    assert pr.gl_ok and ok
    assert (pr.is_prp, pr.res64, pr.old64) == (isp, r64, o64) == (s.is_prp, s.res64, s.old64)
    assert pr.pkey == s.pkey
    assert ck is not None and ck == s.ckey


def test_tampered_proof_is_caught(oracle, tmp_path):
    b, n, depth = 1_000_002, 10, 2
    t = oracle.OracleTransform(b, n, 3 + (1 << depth))
    pr = pf.proof(t, b, n, depth, str(tmp_path / "p.proof"))
    raw = bytearray(open(tmp_path / "p.proof", "rb").read())
    N = 1 << n
    # change one digit of mu[1] (after version, depth and mu[0]), then repair the CRC
    off = 8 + (8 + 4 * N) + 8 + 40
    raw[off] = (raw[off] + 1) % 200
    body = bytes(raw[:-4])
    open(tmp_path / "q.proof", "wb").write(body)
    with pf.GFile(str(tmp_path / "r.proof"), "wb") as f:
        f.write(body)
        f.write_crc32()
    s = pf.server(oracle.OracleTransform(b, n, 4), b, n, str(tmp_path / "r.proof"), str(tmp_path / "r.cert"),
                  (5, 20, 7))
    assert s.pkey != pr.pkey
    open(tmp_path / "bad.proof", "wb").write(bytes(raw))       # CRC not repaired
    with pytest.raises(pf.FileError):
        pf.server(oracle.OracleTransform(b, n, 4), b, n, str(tmp_path / "bad.proof"), str(tmp_path / "b.cert"),
                  (5, 20, 7))


# ------------------------------------------------------------------ deterministic test (mode "prime")

from genefer22_b200 import prime as pm


def _jacobi(a: int, n: int) -> int:
    """Textbook Jacobi symbol for odd n > 0, to check kronecker()."""
    a %= n
    r = 1
    while a:
        while a % 2 == 0:
            a //= 2
            if n % 8 in (3, 5):
                r = -r
        a, n = n, a
        if a % 4 == 3 and n % 4 == 3:
            r = -r
        a %= n
    return r if n == 1 else 0


def test_kronecker_matches_jacobi():
    for y in range(1, 400, 2):
        for x in range(0, 200):
            assert pm.kronecker(x, y) == _jacobi(x, y), (x, y)
    assert pm.kronecker(2, 4) == 0


def test_powmod_as_written():
    # arith.h:13-25 multiplies once more by the last square: a^(2^(k+1)) for e = 2^k
    for m in (7, 11, 101):
        for a in range(2, 20):
            for k in range(0, 6):
                assert pm.powmod(a, 1 << k, m) == pow(a, 1 << (k + 1), m)


def test_prime_factors_and_bases():
    assert pm.prime_factors(824) == [2, 103]
    assert pm.prime_factors(2 * 3 * 3 * 5 * 7 * 7 * 101) == [2, 3, 5, 7, 101]
    it = pm.bases(824, 10)
    got = [next(it)[1] for _ in range(6)]
    a2 = pm.first_base(824, 10)
    assert got[0] == a2 and 4 not in got and 9 not in got and got.count(a2) == 1


def test_prime_on_oracle(oracle):
    """824^(2^10)+1 is prime (the smallest even base at n = 10); 826^(2^10)+1
    is composite; both decided through squareMul on the oracle engine."""
    r = pm.prime(oracle.OracleTransform(824, 10), 824, 10)
    assert r.is_prime is True and all(r.cond)
    r = pm.prime(oracle.OracleTransform(826, 10), 826, 10)
    assert r.is_prime is False
