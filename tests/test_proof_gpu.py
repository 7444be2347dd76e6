"""Proof, server and check modes and context resume over the CUDA engine:
keys consistent across the three modes, files byte-identical to the ones the
oracle engine writes, and a run stopped and resumed from its context file
ending where an uninterrupted run ends."""
import pytest

from genefer22_b200 import Transform
from genefer22_b200 import proof as pf

pytestmark = pytest.mark.gpu


def test_chain_kat():
    """src/main.cpp:417-425: 10^9^(2^11)+1 has res64 43C6CC5326E5C77F."""
    b, n, depth = 1_000_000_000, 11, 4
    import tempfile, os
    d = tempfile.mkdtemp()
    pr = pf.proof(Transform(b, n, 3 + (1 << depth)), b, n, depth, os.path.join(d, "a.proof"))
    assert pr.gl_ok and not pr.is_prp and pr.res64 == 0x43C6CC5326E5C77F
    s = pf.server(Transform(b, n, 4), b, n, os.path.join(d, "a.proof"), os.path.join(d, "a.cert"), (33, 77, 4097))
    assert s.pkey == pr.pkey and s.res64 == pr.res64
    assert pf.check(Transform(b, n, 4), b, n, os.path.join(d, "a.cert")) == s.ckey


def test_files_match_oracle(oracle, tmp_path):
    b, n, depth, rnd = 3_000_002, 10, 3, (9, 31, 555)
    g = tmp_path / "gpu"
    o = tmp_path / "cpu"
    g.mkdir(); o.mkdir()
    pg = pf.proof(Transform(b, n, 3 + (1 << depth)), b, n, depth, str(g / "x.proof"))
    po = pf.proof(oracle.OracleTransform(b, n, 3 + (1 << depth)), b, n, depth, str(o / "x.proof"))
    assert pg == po
    assert (g / "x.proof").read_bytes() == (o / "x.proof").read_bytes()
    sg = pf.server(Transform(b, n, 4), b, n, str(g / "x.proof"), str(g / "x.cert"), rnd)
    so = pf.server(oracle.OracleTransform(b, n, 4), b, n, str(o / "x.proof"), str(o / "x.cert"), rnd)
    assert sg == so
    assert (g / "x.cert").read_bytes() == (o / "x.cert").read_bytes()


def test_prp_resumes_from_context(tmp_path):
    b, n, depth = 50_000_002, 12, 3
    ref = pf.proof(Transform(b, n, 3 + (1 << depth)), b, n, depth, str(tmp_path / "ref.proof"))
    from genefer22_b200.exponent import exponent_words, words_to_int, B_GerbiczLi
    w, nb = exponent_words(b, n)
    E = words_to_int(w)
    B_GL, B_PL = B_GerbiczLi(nb), pf.B_PietrzakLi(nb, depth)
    ctx = str(tmp_path / "t.ctx")
    t1 = Transform(b, n, 3 + (1 << depth))
    r = pf.prp(t1, E, B_GL, B_PL, ctx=ctx, save_every=5000, abort_at=nb // 3)
    assert r.status == "aborted" and r.i == nb // 3
    del t1
    t2 = Transform(b, n, 3 + (1 << depth))
    r = pf.prp(t2, E, B_GL, B_PL, ctx=ctx, save_every=5000)
    assert r.status == "done"
    pkey = pf.PL(t2, b, depth, str(tmp_path / "res.proof"))
    assert pkey == ref.pkey
    assert (tmp_path / "res.proof").read_bytes() == (tmp_path / "ref.proof").read_bytes()


@pytest.mark.parametrize("phase", [0, 1])
def test_check_resumes_from_context(tmp_path, phase):
    b, n, depth = 2_000_000_000, 11, 3
    pr = pf.proof(Transform(b, n, 3 + (1 << depth)), b, n, depth, str(tmp_path / "a.proof"))
    s = pf.server(Transform(b, n, 4), b, n, str(tmp_path / "a.proof"), str(tmp_path / "a.cert"), (40, 200, 60000))
    with pf.GFile(str(tmp_path / "a.cert"), "rb") as f:
        f.read_i32(); B = f.read_i32(); pf.read_gint(f, 1 << n, b); p2 = f.read_mpz()
    stop = p2.bit_length() + B // 2 if phase == 0 else p2.bit_length() // 2
    ctx = str(tmp_path / "c.ctx")
    assert pf.check(Transform(b, n, 4), b, n, str(tmp_path / "a.cert"), ctx=ctx, abort_at=stop) is None
    assert pf.check(Transform(b, n, 4), b, n, str(tmp_path / "a.cert"), ctx=ctx) == s.ckey


def test_wrong_certificate_fails(tmp_path):
    b, n, depth = 1_000_002, 11, 2
    pf.proof(Transform(b, n, 3 + (1 << depth)), b, n, depth, str(tmp_path / "a.proof"))
    s = pf.server(Transform(b, n, 4), b, n, str(tmp_path / "a.proof"), str(tmp_path / "a.cert"), (3, 17, 5))
    with pf.GFile(str(tmp_path / "a.cert"), "rb") as f:
        v, B = f.read_i32(), f.read_i32()
        g = pf.read_gint(f, 1 << n, b)
        p2 = f.read_mpz()
    with pf.GFile(str(tmp_path / "b.cert"), "wb") as f:
        f.write_i32(v); f.write_i32(B); pf.write_gint(f, g, b); f.write_mpz(p2 + 1); f.write_crc32()
    ck = pf.check(Transform(b, n, 4), b, n, str(tmp_path / "b.cert"))
    assert ck is not None and ck != s.ckey


# ------------------------------------------------------------------ deterministic test (mode "prime")

from genefer22_b200 import genefer as gf
from genefer22_b200 import prime as pm


def test_prime_on_gpu():
    assert pm.prime(Transform(824, 10), 824, 10).is_prime is True
    assert pm.prime(Transform(16, 10), 16, 10).is_prime is False      # 2^4096 + 1: probable prime to base 2, composite
    assert pm.prime(Transform(150, 11), 150, 11).is_prime is True
    assert pm.prime(Transform(826, 10), 826, 10).is_prime is False


def test_prp_scan_then_prove():
    """Every even b in [8, 1000) at n = 10 that is not a power of two (the
    bases genefer accepts, src/main.cpp:249-253: base 2 is a Fermat liar for
    every 2^(2^k) + 1) through the batch PRP path; each probable prime is then
    proven prime by the deterministic test."""
    bases = [b for b in range(8, 1000, 2) if b & (b - 1)]
    res = gf.quick_batch(bases, 10)
    assert all(r.gl_ok for r in res)
    prp = [r.b for r in res if r.is_prp]
    assert 824 in prp
    for b in prp:
        assert pm.prime(Transform(b, 10), b, 10).is_prime is True, b


def test_prime_resumes_from_context(tmp_path):
    ctx = str(tmp_path / "p.ctx")
    r = pm.prime(Transform(150, 11), 150, 11, ctx=ctx, save_every=2000, abort_at=(1, 7000))
    assert r.is_prime is None
    r = pm.prime(Transform(150, 11), 150, 11, ctx=ctx)
    assert r.is_prime is True
