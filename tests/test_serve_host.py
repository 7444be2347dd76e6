"""Host logic of the uneven-batch, autotuner and serving modules, on the CPU.

The serving loop runs here against a stand-in for ``Batch`` whose slots are
oracle transforms (the restated transformCPUi32), so that admission, the
per-slot block schedule, retirement, the memory budget and the Gerbicz-Li
validator are checked without a GPU."""
import numpy as np
import pytest

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
    assert candidates(12) == [0, 3, 4, 203]
    assert candidates(14) == [0, 3, 4, 5, 6, 203, 204]
    assert candidates(16) == [1, 3, 4, 5, 6, 7, 8, 203, 204, 103, 104]
    assert candidates(18) == [5, 6, 7, 8, 9, 10, 204, 303, 304, 305, 103, 104, 105, 106]
    assert candidates(23) == [10, 305, 306, 307, 106, 107]


def test_budget():
    bu = sv._Budget(10 * sv.table_bytes(15))
    assert bu.take(15, 100)
    assert bu.used == 100 + sv.table_bytes(15)
    assert bu.take(15, 100)                      # tables counted once per size
    assert bu.used == 200 + sv.table_bytes(15)
    assert not bu.take(16, 10 * sv.table_bytes(15))
    bu.give(15, 100)
    bu.give(15, 100)
    assert bu.used == 0 and bu.peak == 200 + sv.table_bytes(15)


# ------------------------------------------------------------------ serving on a stand-in engine

class _FakeGraph:
    def __init__(self, fn):
        self.fn = fn

    def launch(self):
        self.fn()

    def close(self):
        pass


class FakeBatch:
    """Batch semantics over one oracle transform per slot (reg 3 is scratch)."""
    corrupt = None            # (base, block) -> flip a digit of that test's x after that many blocks

    def __init__(self, bases, n, num_regs=3, device=0, stream=None):
        self.oracle = pytest.importorskip("gf_oracle")
        self.bases = np.asarray(bases, dtype=np.uint32).copy()
        self.n, self.size, self.count = int(n), 1 << int(n), len(bases)
        self.slots = [self.oracle.OracleTransform(int(b), self.n, 4) for b in self.bases]
        self.words = [None] * self.count
        self.pos = [-1] * self.count
        self.blocks = [0] * self.count

    def close(self):
        self.slots = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def plan(self):
        return 0

    def widths(self):
        return np.full(self.count, 3, dtype=np.int32)

    def sync(self):
        pass

    def capture(self, fn):
        return _FakeGraph(fn)

    def assign(self, i, b):
        self.slots[i] = self.oracle.OracleTransform(int(b), self.n, 4)
        self.bases[i] = b

    def put(self, i, d, reg=0):
        o = self.slots[i]
        if reg == 0:
            o.setInt(d)
        else:
            o.copy(3, 0); o.setInt(d); o.copy(reg, 0); o.copy(0, 3)

    def get(self, i, reg=0):
        o = self.slots[i]
        if reg == 0:
            return o.getInt()
        o.copy(3, 0); o.copy(0, reg)
        v = o.getInt()
        o.copy(0, 3)
        return v

    def get_all(self, reg=0):
        return np.stack([self.get(i, reg) for i in range(self.count)])

    def set_exponent(self, i, words, nbits):
        self.words[i] = words_to_int(words)
        self.pos[i] = int(nbits) - 1
        self.blocks[i] = 0

    def set(self, a):
        for o in self.slots:
            o.set(a)

    def copy(self, dst, src):
        for o in self.slots:
            o.copy(dst, src)

    def square(self, dup, count=1):
        for o in self.slots:
            for _ in range(count):
                o.squareDup(bool(dup))

    def square_exp(self, count):
        for i, o in enumerate(self.slots):
            for _ in range(count):
                if self.pos[i] < 0:
                    break
                o.squareDup(bool((self.words[i] >> self.pos[i]) & 1))
                self.pos[i] -= 1
            self.blocks[i] += 1
            c = FakeBatch.corrupt
            if c is not None and c[0] == int(self.bases[i]) and c[1] == self.blocks[i]:
                d = o.getInt()
                d[5] = (d[5] + 1) if d[5] < int(self.bases[i]) // 2 else d[5] - 1
                o.setInt(d)

    def init_multiplicand(self, src):
        for o in self.slots:
            o.initMultiplicand(src)

    def mul_into(self, dst):
        for o in self.slots:
            o.copy(3, 0); o.mul(); o.copy(dst, 0)
            if dst != 0:
                o.copy(0, 3)

    def gl_step(self):
        self.init_multiplicand(1)
        self.mul_into(1)


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


@pytest.fixture
def fake_engine(monkeypatch):
    monkeypatch.setattr(sv, "Batch", FakeBatch)
    FakeBatch.corrupt = None
    yield FakeBatch
    FakeBatch.corrupt = None


def test_serve_loop_on_oracle(fake_engine, oracle):
    B = 6
    reqs = _requests(B)
    ns = sorted({r.job.n for r in reqs})
    budget = sum(2 * sv.slot_bytes(n) + sv.table_bytes(n) for n in ns) + 2 * (sv.slot_bytes(10) + 4096)
    srv = sv.Server(B=B, budget_bytes=budget, capacity=lambda n: 2, validate_group=2, keep_digits=True)
    comps = srv.run(reqs, timeout_s=300)
    assert [c.id for c in comps] == [r.id for r in reqs]
    assert srv.stats.completed == len(reqs) and srv.stats.peak_bytes <= budget
    assert srv.budget.used == 0                   # every pool returned its memory
    for r, c in zip(reqs, comps):
        assert c.gl_ok
        assert np.array_equal(c.digits, _oracle_prefix(oracle, r.job, B)), r.id
        res = gint.is_one(c.digits, r.job.b)
        assert (c.is_prp, c.res64, c.old64) == res
        assert c.arrival <= c.admitted <= c.residue_at <= c.validated_at
    st = srv.stats
    assert st.p50 <= st.p99 and st.rate > 0


def test_serve_validator_flags_a_fault(fake_engine):
    """A digit changed between two blocks of one test fails its Gerbicz-Li
    check; the other tests pass."""
    B = 6
    reqs = _requests(B, count=6, seed=9)
    victim = reqs[2].job
    FakeBatch.corrupt = (victim.b, 1)
    srv = sv.Server(B=B, budget_bytes=10**9, capacity=lambda n: 3, validate_group=2, keep_digits=True)
    comps = srv.run(reqs, timeout_s=300)
    for c in comps:
        assert c.gl_ok == (c.b != victim.b), c.id
    assert srv.stats.gl_failures == 1


def test_serve_budget_too_small(fake_engine):
    reqs = _requests(4, count=2)
    with pytest.raises(ValueError):
        sv.Server(B=4, budget_bytes=1000).run(reqs)


def test_packed_range():
    """The packed-digit range the engine enforces (packed_ok in gf_host.cu)."""
    from genefer22_b200.autotune import packed_ok
    assert packed_ok(184393718, 16) and not packed_ok(184393720, 16)
    assert packed_ok(130386048, 18) and not packed_ok(130386050, 18)
    assert not packed_ok(2**20 - 2, 16) and packed_ok(2**20, 16)
    assert not packed_ok(2**28, 12)


def test_serve_packed_pools(fake_engine, oracle, monkeypatch):
    """Pools of packed-range bases take only such bases, general pools take
    every base; each request is served once and correctly."""
    monkeypatch.setattr(sv, "PACKED_POOL_MIN_N", 8)
    B = 6
    reqs = []
    rng = np.random.default_rng(21)
    for i in range(8):
        b = (2_000_002 + 2 * i) if i % 2 == 0 else (1_000 + 2 * i)   # packed range, below it
        reqs.append(sv.Request(i, gf.Job.prefix(b, 9, 2 * B), 0.001 * i))
    srv = sv.Server(B=B, budget_bytes=10**9, capacity=lambda n: 2, validate_group=2, keep_digits=True)
    comps = srv.run(reqs, timeout_s=300)
    assert sorted(c.id for c in comps) == list(range(8))
    for r, c in zip(reqs, comps):
        assert c.gl_ok and np.array_equal(c.digits, _oracle_prefix(oracle, r.job, B))
    # which pools served which bases: packed-only pools never took a small base
    by_pool = {}
    for c in comps:
        by_pool.setdefault(c.pool, set()).add(sv._packed_pool(c.b, 9))
    assert any(kinds == {True} for kinds in by_pool.values())
