"""The engine against golden vectors that the reference's own CPU transform
produced (tests/golden/make_golden.py) for workloads shaped like the five
benchmark configurations, through the path each configuration uses: the
plain transform, a graph-replayed batch (default packed and unpacked plans), an uneven
batch with tuned plans, and the serving loop."""
import json
import os

import numpy as np
import pytest

from genefer22_b200 import Batch, Transform, gint
from genefer22_b200 import genefer as gf
from genefer22_b200.autotune import Autotuner
from genefer22_b200.mixed import MixedBatch
from genefer22_b200.serve import Request, Server

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))["cases"]


def _keys(canon, b):
    _, r64, o64 = gint.is_one(canon, b)
    return f"{r64:016X}", f"{o64:016X}", f"{gint.hash64(canon):016X}"


def _want(c):
    return c["res64"], c["old64"], c["hash64"]


def test_c1_full_tests_plain_path():
    for c in GOLDEN["c1_full_n12"]:
        r = gf.quick(Transform(c["b"], 12))
        assert (r.is_prp, f"{r.res64:016X}", f"{r.old64:016X}", r.gl_ok) == (c["isPrp"], c["res64"], c["old64"], c["gl"])


@pytest.mark.parametrize("plan", [None, 4])
def test_c2_batch_graph(plan):
    cases = GOLDEN["c2_n16_prefix48"]
    jobs = [gf.Job.prefix(c["b"], 16, c["bits"]) for c in cases]
    with Batch([c["b"] for c in cases], 16) as bt:
        if plan is not None:
            bt.set_plan(plan)
        r = gf.BatchPRP(bt, B=8, exps=[j.words_nbits() for j in jobs])
        r.load()
        r.run_prp()
        got = bt.get_all(0)
        r._graph = None
    for i, c in enumerate(cases):
        assert _keys(gint.unbalance(got[i], c["b"]), c["b"]) == _want(c), i


def test_c3_single_large_test():
    c = GOLDEN["c3_n20_prefix40"][0]
    t = Transform(c["b"], 20)
    job = gf.Job.prefix(c["b"], 20, c["bits"])
    gf.prp(t, job.words, job.nbits, 10)
    assert _keys(gint.unbalance(t.getInt(), c["b"]), c["b"]) == _want(c)


def test_c4_uneven_batch():
    cases = GOLDEN["c4_uneven_prefix40"]
    jobs = [gf.Job.prefix(c["b"], c["n"], c["bits"]) for c in cases]
    with MixedBatch(jobs, B=8, tuner=Autotuner(squarings=4, replays=1)) as mb:
        mb.run(validate=False)
        res = mb.residues()
    for c, canon in zip(cases, res):
        assert _keys(canon, c["b"]) == _want(c), (c["b"], c["n"])


def test_c5_serving():
    cases = GOLDEN["c5_serving_prefix48"]
    reqs = [Request(i, gf.Job.prefix(c["b"], c["n"], c["bits"]), 0.01 * i) for i, c in enumerate(cases)]
    srv = Server(B=8, budget_bytes=20 * 10**9, validate_group=1, keep_digits=True)
    comps = srv.run(reqs, timeout_s=900)
    for c, comp in zip(cases, comps):
        assert comp.gl_ok
        assert _keys(comp.digits, c["b"]) == _want(c), c["n"]
