"""Uneven batches, the plan autotuner and the serving loop on the GPU.

Each test's residue must be the same alone, in an uneven batch and in the
serving mix, and equal to the oracle's (restated transformCPUi32) where the
oracle is run."""
import numpy as np
import pytest

from genefer22_b200 import Batch, GfcError, gint
from genefer22_b200 import genefer as gf
from genefer22_b200.autotune import Autotuner, candidates
from genefer22_b200.exponent import words_to_int
from genefer22_b200.mixed import MixedBatch, run_alone, uneven_tests
from genefer22_b200.serve import Server, pool_slot_bytes, serve_requests, slot_bytes, table_bytes

pytestmark = pytest.mark.gpu


def canon(d, b):
    return gint.unbalance(d, b)


def oracle_prefix(oracle, job, B):
    """reg0 of the oracle after genefer's prp loop over the job's exponent."""
    o = oracle.OracleTransform(job.b, job.n)
    oracle.prp(o, words_to_int(job.words), B)
    return canon(o.getInt(), job.b)


def test_assign_changes_base_and_set(oracle):
    """A slot given a new base (other prime set) squares like a fresh test."""
    n = 12
    bt = Batch([1_000_002, 1_999_999_998], n)
    assert list(bt.widths()) == [2, 3]
    bt.assign(0, 1_999_999_990)
    bt.assign(1, 3_000_002)
    assert list(bt.widths()) == [3, 2]
    rng = np.random.default_rng(3)
    digs = []
    for i, b in enumerate(bt.bases):
        d = rng.integers(-(int(b) // 2), int(b) // 2 + 1, size=1 << n).astype(np.int32)
        bt.put(i, d)
        digs.append(d)
    bt.square(True, 3)
    for i, b in enumerate(bt.bases):
        o = oracle.OracleTransform(int(b), n)
        o.setInt(digs[i])
        for _ in range(3):
            o.squareDup(True)
        assert np.array_equal(canon(bt.get(i), int(b)), canon(o.getInt(), int(b)))


def test_graph_refused_after_set_change():
    """Single-CTA graphs launch per prime set: a change of set since capture
    is refused; four-step graphs stay valid."""
    bt = Batch([1_000_002, 1_999_999_998], 12)
    g = bt.capture(lambda: bt.square(False, 2))
    bt.assign(0, 1_000_004)               # same set: still valid
    g.launch()
    bt.assign(0, 1_999_999_990)           # set 0 -> set 1
    with pytest.raises(GfcError):
        g.launch()
    g.close()
    bt4 = Batch([1_000_002, 1_999_999_998], 15)
    g4 = bt4.capture(lambda: bt4.square(False, 2))
    bt4.assign(0, 1_999_999_990)
    g4.launch()
    bt4.sync()
    g4.close()


@pytest.mark.parametrize("n,plan", [(12, 0), (15, None), (16, 4)])
def test_finished_test_sits_out(oracle, n, plan):
    """A test whose exponent ends while the others continue keeps its residue
    (its segment carries are absorbed once), also across Gerbicz-Li updates."""
    jobs = [gf.Job.prefix(1_000_002, n, 40), gf.Job.prefix(1_999_999_998, n, 150)]
    bt = Batch([j.b for j in jobs], n)
    if plan is not None:
        bt.set_plan(plan)
    for i, j in enumerate(jobs):
        bt.set_exponent(i, j.words, j.nbits)
    bt.set(1)
    bt.copy(1, 0)
    bt.square_exp(100)                    # test 0 ends after 40 squarings
    bt.gl_step()
    bt.square_exp(50)
    bt.gl_step()
    for i, j in enumerate(jobs):
        o = oracle.OracleTransform(j.b, n)
        o.set(1)
        e = words_to_int(j.words)
        for k in range(j.nbits - 1, -1, -1):
            o.squareDup(bool((e >> k) & 1))
        assert np.array_equal(canon(bt.get(i, 0), j.b), canon(o.getInt(), j.b)), i


def test_autotuner(tmp_path):
    path = str(tmp_path / "plans.json")
    tu = Autotuner(cache_path=path, squarings=4, replays=2)
    for n in (12, 15):
        bt = Batch([1_000_002] * 4, n)
        r = tu.tune(bt)
        assert r.lr in candidates(n) and bt.plan() == r.lr
        assert set(r.us) <= set(candidates(n)) and len(r.us) >= 2
        assert abs(bt.get(0)).max() == 0
    tu2 = Autotuner(cache_path=path)
    bt = Batch([1_000_002] * 4, 15)
    assert tu2.tune(bt).lr == tu.cache[f"n15_c4_w0"]["lr"]


def test_uneven_batch_alone_vs_mix(oracle):
    """The uneven workload's shape (sizes 12..18, log-uniform b) with short
    exponent prefixes: every residue equals the test run alone, and the
    oracle's for sizes 12 and 13; Gerbicz-Li passes."""
    B = 32
    tests = uneven_tests(count=24, seed=1004)
    tests += [(2_000_000_000 - 2, 12), (1_000_000_000, 17), (50_000_002, 17), (1024, 18)]
    jobs = [gf.Job.prefix(b, n, 3 * B + 7 * (i % 3)) for i, (b, n) in enumerate(tests)]
    with MixedBatch(jobs, B=B, tuner=Autotuner(squarings=4, replays=1)) as mb:
        res = mb.run()
        canon_mix = mb.residues()
        plans = mb.plans()
        assert set(plans) == {j.n for j in jobs}
        assert plans[17] < 200                               # a base outside the packed range
        assert all(r.gl_ok for r in res)
        assert mb.stats.digit_squarings == sum((1 << j.n) * j.nbits for j in jobs)
    checked = 0
    for i, j in enumerate(jobs):
        r, c = run_alone(j, B)
        assert np.array_equal(c, canon_mix[i]), (j.b, j.n)
        assert r.res64 == res[i].res64
        if j.n <= 13 and checked < 4:
            assert np.array_equal(oracle_prefix(oracle, j, B), c)
            checked += 1


def test_uneven_batch_full_kats():
    """Complete tests of sizes 11 and 12 (res64 of src/main.cpp:417-425) in one
    uneven run, among prefixes of larger tests."""
    kats = {(64611980, 11): 0x6E2E19E3382BC8E8, (2000000000, 11): 0x1A16EAEE2487902D,
            (23448336, 12): 0x81CFF004ACE85CAA, (1000000000, 12): 0x4E43A5B93273C649}
    jobs = [gf.Job.full(b, n) for (b, n) in kats]
    jobs += [gf.Job.prefix(50_000_000, 16, 3000), gf.Job.prefix(20_000_000, 18, 3000)]
    with MixedBatch(jobs, B=None) as mb:
        res = mb.run()
    for j, r in zip(jobs, res):
        assert r.gl_ok
        if (j.b, j.n) in kats:
            assert r.res64 == kats[(j.b, j.n)], hex(r.res64)


def test_serve_alone_vs_mix(oracle):
    """Poisson arrivals of sizes 15..17 under a budget that admits only part of
    them at once: each residue equals the test alone, Gerbicz-Li passes, the
    budget holds, and some requests wait for memory."""
    B = 32
    reqs = serve_requests(count=14, rate=200.0, blocks=[2, 3], B=B, seed=1005, ns=(15, 16, 17), big=None)
    ns = (15, 16, 17)
    budget = (sum(2 * slot_bytes(n, B + 96) + table_bytes(n) for n in ns)   # checkers, root tables
              + 2 * 2 * pool_slot_bytes(17, B))                               # two pools of two slots
    srv = Server(B=B, budget_bytes=budget, capacity=lambda n: 2, validate_group=2, keep_digits=True)
    comps = srv.run(reqs, timeout_s=600)
    st = srv.stats
    assert st.completed == len(reqs)
    assert st.peak_bytes <= budget
    assert st.pools_created >= 3                # pools closed and reopened within the budget
    assert all(c.gl_ok for c in comps)
    assert st.mean_wait > 0
    for r, c in zip(reqs, comps):
        assert c.id == r.id and c.residue_at >= c.admitted >= r.arrival
        _, alone = run_alone(r.job, B)
        assert np.array_equal(alone, c.digits), (r.job.b, r.job.n)
    j = min((r.job for r in reqs), key=lambda j: j.n)
    assert np.array_equal(oracle_prefix(oracle, j, B), next(c.digits for c in comps if c.b == j.b))


def test_serve_with_large_test():
    """A size-23 test (8,388,608 digits) served among smaller ones."""
    B = 16
    reqs = serve_requests(count=6, rate=50.0, blocks=[2], B=B, seed=7, ns=(15, 20), big=23)
    srv = Server(B=B, budget_bytes=8 * 10**9, validate=True, validate_group=1, keep_digits=True)
    comps = srv.run(reqs, timeout_s=900)
    assert all(c.gl_ok for c in comps)
    big = [c for c in comps if c.n == 23]
    assert len(big) == 1
    r = next(r for r in reqs if r.job.n == 23)
    _, alone = run_alone(r.job, B)
    assert np.array_equal(alone, big[0].digits)


def test_admission_leaves_other_pools_running(oracle):
    """Admitting a test into one pool (gfc_batch_admit) neither allocates device
    memory nor waits for another pool's graph in flight: right after the call
    returns, the other pool's replay is still running; the admitted test then
    squares like a fresh test."""
    import torch
    B = 8
    big = Batch([30_000_002] * 2, 20)
    g = big.capture(lambda: big.square(False, 400))        # about 20 ms of device work
    small = Batch([1_000_002, 1_999_999_998], 12)
    small.reserve(4 * B)
    job = gf.Job.prefix(2_000_000_000 - 2, 12, 3 * B)
    s_big = torch.cuda.ExternalStream(big.stream)
    ev = torch.cuda.Event()
    g.launch()
    ev.record(s_big)
    free0 = torch.cuda.mem_get_info(0)[0]
    small.admit(1, job.b, job.words, job.nbits)            # prime set changes too (2 -> 3 primes)
    assert not ev.query(), "admission waited for the other pool's graph"
    assert torch.cuda.mem_get_info(0)[0] >= free0
    small.square_exp(job.nbits)
    assert np.array_equal(canon(small.get(1, 0), job.b), oracle_prefix(oracle, job, 10**9))
    g.close()


def test_native_server_reports_plans_and_stats():
    """The native loop's completions carry the pool's plan and the stats its
    counters: blocks run, pools opened, peak memory within the budget."""
    B = 16
    reqs = serve_requests(count=6, rate=100.0, blocks=[2], B=B, seed=3, ns=(15, 16), big=None)
    srv = Server(B=B, budget_bytes=4 * 10**9, validate_group=2, keep_digits=False)
    comps = srv.run(reqs, timeout_s=300)
    assert all(c.gl_ok for c in comps)
    assert all(c.plan in candidates(c.n) for c in comps)
    st = srv.stats
    assert st.blocks_run >= 2 and 1 <= st.pools_created and st.peak_bytes <= 4 * 10**9
    assert st.p50 <= st.p99
