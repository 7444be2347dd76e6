"""The oracle (restated transformCPUi32) against golden vectors that the
reference's own CPU transform produced (tests/golden/make_golden.py), and
the exponent prefixes the product computes without forming E."""
import json
import os

import numpy as np
import pytest

from genefer22_b200 import genefer as gf
from genefer22_b200 import gint
from genefer22_b200.exponent import words_to_int

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))["cases"]


def _oracle_prefix(oracle, c):
    job = gf.Job.prefix(c["b"], c["n"], c["bits"])
    assert job.nbits == c["bits"]
    o = oracle.OracleTransform(c["b"], c["n"])
    o.set(1)
    e = words_to_int(job.words)
    for i in range(job.nbits - 1, -1, -1):
        o.squareDup(bool((e >> i) & 1))
    canon = gint.unbalance(o.getInt(), c["b"])
    _, r64, o64 = gint.is_one(canon, c["b"])
    return f"{r64:016X}", f"{o64:016X}", f"{gint.hash64(canon):016X}"


def _cheap():
    out = [c for c in GOLDEN["c4_uneven_prefix40"] if c["n"] <= 13][:6]
    out += GOLDEN["c2_n16_prefix48"][:2] + [c for c in GOLDEN["c5_serving_prefix48"] if c["n"] == 15]
    return out


@pytest.mark.parametrize("c", _cheap(), ids=lambda c: f"n{c['n']}-b{c['b']}")
def test_oracle_matches_reference_golden(oracle, c):
    assert _oracle_prefix(oracle, c) == (c["res64"], c["old64"], c["hash64"])


def test_c5_states_wrap():
    """Each configuration-5 case squares long enough that the state 2^e (e the exponent
    prefix, e >= 2^(bits-1)) exceeds b^N and wraps modulo b^N + 1: the later squarings
    work on dense digits, with carries across the whole register."""
    import math
    for c in GOLDEN["c5_serving_prefix48"]:
        assert 2 ** (c["bits"] - 1) > (1 << c["n"]) * math.log2(c["b"]) * 2 ** 16, c["n"]


def test_golden_shapes():
    assert len(GOLDEN["c2_n16_prefix48"]) == 64 and {c["n"] for c in GOLDEN["c2_n16_prefix48"]} == {16}
    assert {c["n"] for c in GOLDEN["c5_serving_prefix48"]} == set(range(15, 24))
    assert all(c["gl"] and not c["isPrp"] for c in GOLDEN["c1_full_n12"])
