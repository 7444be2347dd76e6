"""Golden vectors from the reference's own CPU transform.

transformCPUi32 (src/transformCPUi32.h), compiled from the genefer sources
into oracle/_ref/libgfref.so by oracle/Makefile, squares seeded inputs shaped
like the five benchmark configurations; the results go to golden.json beside
this script.  Exponents come from GMP (libgmp.so.10, as genefer computes
them, src/genefer.h:1476); a prefix of k bits is E >> (|E| - k), the state of
genefer's prp loop after k squarings (src/genefer.h:505-549).

    python tests/golden/make_golden.py      # where the genefer sources are

Each record: b, n, bits (squarings), res64 / old64 / hash64 of the canonical
residue (gint::isOne, gint::gethash64, src/gint.h:169-225); full tests also
isPrp and the Gerbicz-Li check of genefer::quick (src/genefer.h:736-748).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import gf_oracle as G                                     # noqa: E402
from genefer22_b200.exponent import exponent_words, words_to_int   # noqa: E402
from genefer22_b200.mixed import uneven_tests             # noqa: E402


def prefix_int(b, n, bits):
    w, nb = exponent_words(b, n)
    e = words_to_int(w)
    k = min(bits, nb)
    return e >> (nb - k), k


def run_prefix(b, n, bits):
    e, k = prefix_int(b, n, bits)
    t = G.RefTransform(b, n, impl="i32")
    t.set(1)
    t.run_squarings(np.array([(e >> i) & 1 for i in range(k - 1, -1, -1)], dtype=np.uint8))
    canon = G.unbalance(t.getInt(), b)
    _, r64, o64 = G.is_one(canon, b)
    return {"b": b, "n": n, "bits": k, "res64": f"{r64:016X}", "old64": f"{o64:016X}", "hash64": f"{G.hash64(canon):016X}"}


def run_full(b, n):
    t = G.RefTransform(b, n, impl="i32")
    is_prp, r64, o64, ok = G.quick(t, b, n)
    return {"b": b, "n": n, "isPrp": bool(is_prp), "res64": f"{r64:016X}", "old64": f"{o64:016X}", "gl": bool(ok)}


def main():
    out = {"source": "reference transformCPUi32 (oracle/_ref), GMP exponents", "cases": {}}
    # configuration 1: full tests at n = 12, b even uniform in [1024, 2e6], seed 1001
    rng = np.random.default_rng(1001)
    bs = [int(x) * 2 for x in rng.integers(512, 10**6 + 1, size=2)]
    out["cases"]["c1_full_n12"] = [run_full(b, 12) for b in bs]
    print("c1", flush=True)
    # configuration 2: 64 tests at n = 16, b even uniform in [1e6, 1e8], seed 1002; 48 squarings each
    rng = np.random.default_rng(1002)
    bs = (rng.integers(10**6 // 2, 10**8 // 2 + 1, size=64) * 2).tolist()
    out["cases"]["c2_n16_prefix48"] = [run_prefix(int(b), 16, 48) for b in bs]
    print("c2", flush=True)
    # configuration 3: n = 20, b even uniform in [1e6, 5e7], seed 1003; 40 squarings
    rng = np.random.default_rng(1003)
    b = int(rng.integers(5 * 10**5, 25 * 10**6)) * 2
    out["cases"]["c3_n20_prefix40"] = [run_prefix(b, 20, 40)]
    print("c3", flush=True)
    # configuration 4: the first 48 tests of the uneven workload (seed 1004); 40 squarings each
    out["cases"]["c4_uneven_prefix40"] = [run_prefix(b, n, 40) for b, n in uneven_tests(256, seed=1004)[:48]]
    print("c4", flush=True)
    # configuration 5: n = 15..23 at the per-n limits' scale (seed 1005); 48 squarings each.  The
    # state after k squarings from 1 is 2^e with e < 2^k, so k >= 28 is needed before it
    # exceeds b^N at n = 23 and wraps; the last 20 or more squarings then work on dense
    # states with carries across the whole register.
    rng = np.random.default_rng(1005)
    lim = {15: 2_000_000_000, 16: 1_500_000_000, 17: 10**9, 18: 10**9, 19: 70_000_000, 20: 55_000_000,
           21: 45_000_000, 22: 35_000_000, 23: 25_000_000}
    cases = []
    for n in range(15, 24):
        b = int(rng.integers(1024, lim[n])) & ~1
        cases.append(run_prefix(b, n, 48))
        print("c5", n, flush=True)
    out["cases"]["c5_serving_prefix48"] = cases
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
