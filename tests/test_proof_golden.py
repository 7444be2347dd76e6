"""genefer22_b200.proof against genefer's OWN proof, server and check modes.

The fixtures under tests/golden/proof/ were written by genefer itself
(src/genefer.h:479-1099, driven by oracle/_ref/genefer_harness;
tests/golden/make_proof_golden.py): its proof file, its certificate and the
keys its modes printed.  The restated modes must write the same bytes and
find the same keys: on the oracle engine here (CPU), and on the CUDA engine
(marked gpu)."""
import json
import os

import pytest

from genefer22_b200 import proof as pf

HERE = os.path.join(os.path.dirname(__file__), "golden", "proof")
KEYS = json.load(open(os.path.join(HERE, "keys.json")))["cases"]


def _check_case(make, name, tmp_path):
    c = KEYS[name]
    b, n, depth = c["b"], c["n"], c["depth"]
    src = os.path.join(HERE, name)
    # Proof mode: the proof file and pkey genefer wrote
    pr = pf.proof(make(b, n, 3 + (1 << depth)), b, n, depth, str(tmp_path / "g.proof"))
    assert (pr.is_prp, f"{pr.res64:016X}", f"{pr.old64:016X}", f"{pr.pkey:016X}") == \
        (c["isPrp"], c["res64"], c["old64"], c["pkey"])
    assert pr.gl_ok
    assert (tmp_path / "g.proof").read_bytes() == open(os.path.join(src, "g.proof"), "rb").read()
    # Server mode on genefer's proof file, with the random exponents genefer drew
    s = pf.server(make(b, n, 4), b, n, os.path.join(src, "g.proof"), str(tmp_path / "g.cert"), tuple(c["rnd"]))
    assert (f"{s.pkey:016X}", f"{s.ckey:016X}", f"{s.res64:016X}") == (c["pkey"], c["ckey"], c["res64"])
    assert (tmp_path / "g.cert").read_bytes() == open(os.path.join(src, "g.cert"), "rb").read()
    # Check mode on genefer's certificate
    assert f"{pf.check(make(b, n, 4), b, n, os.path.join(src, 'g.cert')):016X}" == c["ckey"]


@pytest.mark.parametrize("name", sorted(KEYS))
def test_oracle_engine_matches_genefer(oracle, name, tmp_path):
    _check_case(lambda b, n, r: oracle.OracleTransform(b, n, r), name, tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(KEYS))
def test_cuda_engine_matches_genefer(name, tmp_path):
    from genefer22_b200 import Transform
    _check_case(lambda b, n, r: Transform(b, n, r), name, tmp_path)
