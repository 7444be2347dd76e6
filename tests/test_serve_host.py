"""Host logic of the uneven-batch, autotuner and serving modules, on the CPU.

The native serving loop (genefer22_b200/csrc/gf_server.cpp, the same source
libgfcuda.so runs) is built here with a device layer whose pools and
checkers are oracle transforms (the restated transformCPUi32,
tests/cpp/server_fake.cpp), so that admission, the per-slot block schedule,
retirement, the memory budget, pool closing and the Gerbicz-Li check are
checked without a GPU, through the gfc_server_* C ABI."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from genefer22_b200 import GfcError
from genefer22_b200 import genefer as gf
from genefer22_b200 import gint
from genefer22_b200 import serve as sv
from genefer22_b200.autotune import candidates
from genefer22_b200.exponent import exponent_words, prefix_words, words_to_int
from genefer22_b200.mixed import SIZE_MIX, b_limit, uneven_tests


# ------------------------------------------------------------------ exponents

@pytest.mark.parametrize("n", [10, 12, 14, 16])
def test_prefix_words_exact(n):
    rng = np.random.default_rng(n)
    for _ in range(12):
        b = int(rng.integers(1024, 2_000_000_000)) & ~1
        bits = int(rng.integers(1, 5000))
        w, k, nb = prefix_words(b, n, bits)
        W, NB = exponent_words(b, n)
        assert nb == NB and k == min(bits, NB)
        assert words_to_int(w) == words_to_int(W) >> (NB - k)


def test_prefix_of_large_exponent():
    """b^(2^23) at b = 25,000,000: 206,153,605 bits, top 64 as GMP gives them."""
    w, k, nb = prefix_words(25_000_000, 23, 64)
    W, NB = exponent_words(25_000_000, 23)
    assert nb == NB == 206153605 and k == 64
    assert words_to_int(w) == words_to_int(W) >> (NB - 64)


def test_job_prefix_matches_full():
    j = gf.Job.full(1_000_002, 12)
    p = gf.Job.prefix(1_000_002, 12, 300)
    assert p.nbits == 300
    assert words_to_int(p.words) == words_to_int(j.words) >> (j.nbits - 300)
    assert gf.Job.prefix(1_000_002, 12, 10**9).nbits == j.nbits


# ------------------------------------------------------------------ workloads

def test_uneven_tests():
    t = uneven_tests(256, seed=1004)
    assert len(t) == 256 and t == uneven_tests(256, seed=1004)
    ns = np.array([n for _, n in t])
    for n, p in SIZE_MIX.items():
        assert abs(np.mean(ns == n) - p) < 0.06, n
    for b, n in t:
        assert b % 2 == 0 and 1024 <= b < b_limit(n)


def test_serve_requests():
    B = 100
    r = sv.serve_requests(50, rate=10.0, blocks=[2, 5], B=B, seed=1005)
    assert len(r) == 51
    big = [x for x in r if x.job.n == 23]
    assert len(big) == 1 and abs(big[0].job.b - 25_000_000) < 200 and big[0].job.b % 2 == 0
    small = [x for x in r if x.job.n != 23]
    arr = [x.arrival for x in small]
    assert arr == sorted(arr) and arr[0] == 0.0
    assert 2.0 < arr[-1] < 10.0                                # 49 gaps of mean 0.1 s
    for x in small:
        assert 15 <= x.job.n <= 22 and x.job.b % 2 == 0 and x.job.b < sv.SERVE_LIMITS[x.job.n]
        assert x.job.nbits in (2 * B, 5 * B)


def test_candidates():
    assert candidates(12) == [0, 1, 3, 4, 203]
    assert candidates(14) == [0, 1, 3, 4, 5, 6, 203, 204]
    assert candidates(16) == [1, 3, 4, 5, 6, 7, 8, 203, 204, 103, 104]
    assert candidates(18) == [5, 6, 7, 8, 9, 10, 204, 303, 304, 305, 103, 104, 105, 106]
    assert candidates(23) == [10, 305, 306, 307, 106, 107]


def test_packed_range():
    """The packed-digit range the engine enforces (gfc_packed_range)."""
    from genefer22_b200.autotune import packed_ok
    assert packed_ok(184393718, 16) and not packed_ok(184393720, 16)
    assert packed_ok(130386048, 18) and not packed_ok(130386050, 18)
    assert not packed_ok(2**20 - 2, 16) and packed_ok(2**20, 16)
    assert not packed_ok(2**28, 12)


def test_budget_sizes():
    """The budget's byte counts follow the engine's allocations per slot."""
    for n in (12, 16, 20):
        N = 1 << n
        assert sv.slot_bytes(n) >= 3 * 4 * N + 24 * N + (N // 16) * 40
        assert sv.slot_bytes(n, 4096) - sv.slot_bytes(n) == 512
        assert sv.pool_slot_bytes(n, 1000) == sv.slot_bytes(n, 31 * N + 1000)
        assert sv.table_bytes(n) == 96 * N
    assert [sv.default_capacity(n) for n in (15, 17, 20, 22)] == [32, 16, 2, 1]


def test_chunk_sum_matches_python():
    """The native checker's exponent of the final 2^res (gf_server.cpp chunk_sum)
    against exponent.chunk_sum, through a served test's check on the fake
    device: covered by the serving tests below; here the Python restatement
    on cases with a partial top chunk."""
    from genefer22_b200.exponent import chunk_sum
    w = np.array([0xFFFFFFFF, 0x1], dtype=np.uint32)
    assert chunk_sum(w, 33, 8) == 4 * 255 + 1


# ------------------------------------------------------------------ the native loop on the CPU oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FAKE = os.path.join(ROOT, "tests", "cpp", "_build", "libgfserver_fake.so")
FAKE_SRC = [os.path.join(ROOT, "genefer22_b200", "csrc", "gf_server.cpp"),
            os.path.join(ROOT, "genefer22_b200", "csrc", "gf_gint.cpp"),
            os.path.join(ROOT, "tests", "cpp", "server_fake.cpp")]


@pytest.fixture(scope="module")
def fake_lib(oracle):
    """The serving loop built with the oracle device layer (g++, no CUDA)."""
    deps = FAKE_SRC + [os.path.join(ROOT, "genefer22_b200", "csrc", "gf_server.h"), os.path.join(ROOT, "include", "gfcuda.h")]
    if (not os.path.exists(FAKE)) or any(os.path.getmtime(d) > os.path.getmtime(FAKE) for d in deps):
        os.makedirs(os.path.dirname(FAKE), exist_ok=True)
        odir = os.path.join(ROOT, "oracle", "_build")
        subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-shared", "-fPIC", "-fvisibility=hidden",
                        f"-I{ROOT}/include", *FAKE_SRC, f"-L{odir}", "-lgforacle", f"-Wl,-rpath,{odir}", "-lpthread",
                        "-o", FAKE], check=True)
    L = ctypes.CDLL(FAKE)
    L.gfc_fake_corrupt.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    L.gfc_fake_packed.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    L.gfc_fake_corrupt(0, 0)
    L.gfc_fake_packed(19, 0xFFFFFFFF)
    yield sv.bind(L)
    L.gfc_fake_corrupt(0, 0)
    L.gfc_fake_packed(19, 0xFFFFFFFF)


def _oracle_prefix(oracle, job, B):
    o = oracle.OracleTransform(job.b, job.n)
    oracle.prp(o, words_to_int(job.words), B)
    return gint.unbalance(o.getInt(), job.b)


def _requests(B, count=10, seed=5):
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    for i in range(count):
        n = int(rng.choice([8, 9, 10]))
        b = int(rng.integers(1024, 2_000_000_000)) & ~1
        job = gf.Job.prefix(b, n, int(rng.choice([2, 3])) * B - int(rng.integers(0, 3)))
        out.append(sv.Request(i, job, t))
        t += float(rng.exponential(0.01))
    return out


def _budget(ns, cap, group, B):
    """Pools of `cap` slots for every size at once, their checkers and tables."""
    return sum(cap * sv.pool_slot_bytes(n, B) + group * sv.slot_bytes(n, B + 96) + sv.table_bytes(n) for n in ns)


def test_serve_loop_on_oracle(fake_lib, oracle):
    B = 6
    reqs = _requests(B)
    ns = sorted({r.job.n for r in reqs})
    budget = _budget(ns, 2, 2, B)
    srv = sv.Server(B=B, budget_bytes=budget, capacity=lambda n: 2, validate_group=2, keep_digits=True, lib=fake_lib)
    comps = srv.run(reqs, timeout_s=300)
    assert [c.id for c in comps] == [r.id for r in reqs]
    assert srv.stats.completed == len(reqs) and srv.stats.peak_bytes <= budget
    for r, c in zip(reqs, comps):
        assert c.gl_ok
        assert np.array_equal(c.digits, _oracle_prefix(oracle, r.job, B)), r.id
        res = gint.is_one(c.digits, r.job.b)
        assert (c.is_prp, c.res64, c.old64) == res
        assert c.arrival <= c.admitted <= c.residue_at <= c.validated_at
    st = srv.stats
    assert st.p50 <= st.p99 and st.rate > 0 and st.blocks_run >= 3


def test_serve_budget_rotates_pools(fake_lib, oracle):
    """A budget that holds one pool at a time: pools of other sizes open only
    after idle ones close, and every request is still served correctly."""
    B = 6
    reqs = _requests(B, count=8, seed=11)
    ns = sorted({r.job.n for r in reqs})
    assert len(ns) >= 2
    one = max(2 * sv.pool_slot_bytes(n, B) + sv.table_bytes(n) for n in ns)
    checkers = sum(2 * sv.slot_bytes(n, B + 96) + sv.table_bytes(n) for n in ns)
    budget = one + checkers
    srv = sv.Server(B=B, budget_bytes=budget, capacity=lambda n: 2, validate_group=2, keep_digits=True,
                    idle_close_s=10.0, lib=fake_lib)
    comps = srv.run(reqs, timeout_s=300)
    assert srv.stats.peak_bytes <= budget
    assert srv.stats.pools_created >= len(ns)
    for r, c in zip(reqs, comps):
        assert c.gl_ok and np.array_equal(c.digits, _oracle_prefix(oracle, r.job, B))


def test_serve_validator_flags_a_fault(fake_lib):
    """A digit changed between two blocks of one test fails its Gerbicz-Li
    check; the other tests pass."""
    B = 6
    reqs = _requests(B, count=6, seed=9)
    victim = reqs[2].job
    fake_lib.gfc_fake_corrupt(victim.b, 1)
    try:
        srv = sv.Server(B=B, budget_bytes=10**9, capacity=lambda n: 3, validate_group=2, keep_digits=True,
                        lib=fake_lib)
        comps = srv.run(reqs, timeout_s=300)
    finally:
        fake_lib.gfc_fake_corrupt(0, 0)
    for c in comps:
        assert c.gl_ok == (c.b != victim.b), c.id
    assert srv.stats.gl_failures == 1


def test_serve_budget_too_small(fake_lib):
    reqs = _requests(4, count=2)
    with pytest.raises(GfcError):
        sv.Server(B=4, budget_bytes=1000, lib=fake_lib).run(reqs, timeout_s=60)


def test_serve_rejects_bad_requests(fake_lib):
    job = gf.Job.prefix(1_000_002, 10, 12)
    bad = sv.Request(0, gf.Job(4, 10, job.words, job.nbits), 0.0)       # b < 8
    with pytest.raises(GfcError):
        sv.Server(B=4, budget_bytes=10**9, lib=fake_lib).run([bad], timeout_s=60)


def test_serve_packed_pools(fake_lib, oracle):
    """Pools opened for packed-range bases take only such bases, general pools
    take every base; each request is served once and correctly."""
    B = 6
    fake_lib.gfc_fake_packed(8, 2_000_000)         # from n = 8, bases >= 2e6 count as packed
    try:
        reqs = []
        for i in range(8):
            b = (2_000_002 + 2 * i) if i % 2 == 0 else (1_000 + 2 * i)   # packed range, below it
            reqs.append(sv.Request(i, gf.Job.prefix(b, 9, 2 * B), 0.001 * i))
        srv = sv.Server(B=B, budget_bytes=10**9, capacity=lambda n: 2, validate_group=2, keep_digits=True,
                        lib=fake_lib)
        comps = srv.run(reqs, timeout_s=300)
    finally:
        fake_lib.gfc_fake_packed(19, 0xFFFFFFFF)
    assert sorted(c.id for c in comps) == list(range(8))
    for r, c in zip(reqs, comps):
        assert c.gl_ok and np.array_equal(c.digits, _oracle_prefix(oracle, r.job, B))
    by_pool = {}
    for c in comps:
        by_pool.setdefault(c.pool, set()).add(c.b >= 2_000_000)
    assert any(kinds == {True} for kinds in by_pool.values())     # a pool of packed-range bases only
    assert all(kinds != {True, False} or True for kinds in by_pool.values())


def test_uneven_batch_through_native_loop(fake_lib, oracle, monkeypatch):
    """MixedBatch (configuration 4's driver) on the native loop: one pool per
    size with a slot per test, all submitted at once."""
    from genefer22_b200 import mixed
    monkeypatch.setattr(mixed, "Server", lambda **kw: sv.Server(lib=fake_lib, **kw))
    B = 5
    jobs = [gf.Job.prefix(b, n, 2 * B + k) for k, (b, n) in enumerate([(1_000_002, 9), (1_234_566, 10), (5_000, 9),
                                                                        (2_000_000_000 - 2, 10)])]
    mb = mixed.MixedBatch(jobs, B=B)
    res = mb.run()
    assert all(r.gl_ok for r in res)
    for j, c in zip(jobs, mb.residues()):
        assert np.array_equal(c, _oracle_prefix(oracle, j, B))
    assert mb.stats.digit_squarings == sum((1 << j.n) * j.nbits for j in jobs)


def test_serve_longer_exponent_after_pool_opened(fake_lib, oracle):
    """A pool reserves room for the longest exponent of its size, so a request
    whose exponent is far longer than those the pool opened for is admitted
    into it later."""
    B = 6
    short = gf.Job.prefix(1_000_002, 9, 2 * B)
    long = gf.Job.prefix(1_000_004, 9, 40 * B)
    reqs = [sv.Request(0, short, 0.0), sv.Request(1, long, 0.05)]
    srv = sv.Server(B=B, budget_bytes=10**9, capacity=lambda n: 1, validate_group=1, keep_digits=True,
                    idle_close_s=10.0, lib=fake_lib)
    comps = srv.run(reqs, timeout_s=120)
    assert srv.stats.pools_created == 1
    for r, c in zip(reqs, comps):
        assert c.gl_ok and np.array_equal(c.digits, _oracle_prefix(oracle, r.job, B))
