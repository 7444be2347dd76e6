"""Cluster-resident squaring (plan 1, 12 <= n <= 17): one thread-block cluster
per test, the state in distributed shared memory across many squarings
(eight CTAs with plane-split passes up to n = 14, rows of 2^13 above).
Results must equal the oracle's (restated transformCPUi32) and the four-step
plan's, digit for digit after canonicalisation."""
import numpy as np
import pytest

from genefer22_b200 import Batch, Transform, gint
from genefer22_b200 import genefer as gf
from genefer22_b200.exponent import words_to_int

pytestmark = pytest.mark.gpu

PLAN_CLUSTER = 1


def canon(d, b):
    return gint.unbalance(d, b)


def rand_digits(rng, b, N):
    return rng.integers(-(b // 2), b // 2 + 1, size=N).astype(np.int32)


@pytest.mark.parametrize("n", [12, 13, 14, 15, 16, 17])
@pytest.mark.parametrize("b", [2_000_002, 1_999_999_998, 1024])
def test_cluster_squarings_vs_oracle(oracle, n, b):
    rng = np.random.default_rng(n * 7 + b % 11)
    t = Transform(b, n)
    t.batch.set_plan(PLAN_CLUSTER)
    assert t.batch.plan() == PLAN_CLUSTER
    o = oracle.OracleTransform(b, n)
    d = rand_digits(rng, b, 1 << n)
    t.setInt(d)
    o.setInt(d)
    for k in range(3):
        dup = (k == 1)
        t.squareDup(dup)
        o.squareDup(dup)
        g = t.getInt()
        assert np.abs(g).max() <= b // 2 + 1
        assert np.array_equal(canon(g, b), canon(o.getInt(), b)), f"square {k}"
    # products run on the four-step plan, squarings after them on the cluster plan
    t.copy(1, 0); o.copy(1, 0)
    t.squareDup(False); o.squareDup(False)
    t.mul(1); o.mul(1)
    t.squareDup(True); o.squareDup(True)
    assert np.array_equal(canon(t.getInt(), b), canon(o.getInt(), b)), "mul"


def _run_block(bases, n, plan, B, nblocks, words_nbits):
    bt = Batch(bases, n)
    bt.set_plan(plan)
    runner = gf.BatchPRP(bt, B=B, exps=words_nbits)
    runner.load()
    bt.square_exp(runner.schedule()[0])
    bt.gl_step()
    g = runner.block_graph()
    for _ in range(nblocks):
        g.launch()
    pos = bt.get_pos()
    r0, r1 = bt.get_all(0), bt.get_all(1)
    runner._graph = None
    bt.close()
    return pos, r0, r1


@pytest.mark.parametrize("n,count", [(15, 150), (16, 40), (17, 9)])
def test_cluster_batch_graph_matches_four_step(n, count):
    """Graph-replayed Gerbicz-Li blocks with more tests than resident
    clusters (the persistent grid loops over tests), both prime sets."""
    rng = np.random.default_rng(n)
    bases = [int(x) & ~1 for x in rng.integers(1_000_000, 100_000_000, size=count)]
    B = 24
    exps = [gf.Job.prefix(b, n, 5 * B).words_nbits() for b in bases]
    got = _run_block(bases, n, PLAN_CLUSTER, B, 2, exps)
    ref = _run_block(bases, n, n - 12, B, 2, exps)
    assert np.array_equal(got[0], ref[0])
    for i, b in enumerate(bases):
        assert np.array_equal(canon(got[1][i], b), canon(ref[1][i], b)), i
        assert np.array_equal(canon(got[2][i], b), canon(ref[2][i], b)), i


def test_cluster_prefix_vs_oracle(oracle):
    n, B = 16, 16
    jobs = [gf.Job.prefix(50_000_000, n, 3 * B), gf.Job.prefix(3_000_000, n, 2 * B + 5)]
    bt = Batch([j.b for j in jobs], n)
    bt.set_plan(PLAN_CLUSTER)
    runner = gf.BatchPRP(bt, B=B, exps=[j.words_nbits() for j in jobs])
    runner.load()
    runner.run_prp()
    got = bt.get_all(0)
    for i, j in enumerate(jobs):
        o = oracle.OracleTransform(j.b, n)
        oracle.prp(o, words_to_int(j.words), B)
        assert np.array_equal(canon(got[i], j.b), canon(o.getInt(), j.b)), i


def test_cluster_finished_test_sits_out(oracle):
    n = 16
    jobs = [gf.Job.prefix(1_000_002, n, 40), gf.Job.prefix(1_999_999_998, n, 90)]
    bt = Batch([j.b for j in jobs], n)
    bt.set_plan(PLAN_CLUSTER)
    for i, j in enumerate(jobs):
        bt.set_exponent(i, j.words, j.nbits)
    bt.set(1)
    bt.copy(1, 0)
    bt.square_exp(60)
    bt.gl_step()
    bt.square_exp(50)
    assert list(bt.get_pos()) == [-1, -1]
    for i, j in enumerate(jobs):
        o = oracle.OracleTransform(j.b, n)
        o.set(1)
        e = words_to_int(j.words)
        for k in range(j.nbits - 1, -1, -1):
            o.squareDup(bool((e >> k) & 1))
        assert np.array_equal(canon(bt.get(i, 0), j.b), canon(o.getInt(), j.b)), i
