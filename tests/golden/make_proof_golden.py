"""Proof, certificate and key fixtures from genefer's OWN proof, server and
check modes (src/genefer.h:479-1099, run by genefer::check, :1376-1600).

oracle/_ref/genefer_harness (built by oracle/Makefile from the reference
sources where they lie) runs genefer's Proof, Server and Check modes on the
reference's i32 CPU transform with a fixed seed for the server's random
exponents.  For each case this script keeps genefer's proof file and
certificate under proof/<name>/ and writes proof/keys.json: res64, old64,
pkey (Proof and Server modes), ckey (Server and Check modes), and the
server's random exponents (rnd1, rnd2, rnd3).

    python tests/golden/make_proof_golden.py      # where the genefer sources are
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "genefer_harness")

# (name, b, n, depth, seed time): small sizes, the i32 transform is single-threaded.
# 10^9 at n = 11 is the main.cpp known-answer base (src/main.cpp:417-425).
CASES = [("b3000002_n10_d3", 3_000_002, 10, 3, 1_700_000_000),
         ("b1000000000_n11_d4", 1_000_000_000, 11, 4, 1_700_000_123),
         ("b150_n10_d2", 150, 10, 2, 1_700_000_456)]

KEY = re.compile(r"(res64|old64|pkey|ckey) = ([0-9A-F]{16})")


def main():
    if not os.path.exists(HARNESS):
        sys.exit("oracle/_ref/genefer_harness is not built (make -C oracle ref)")
    out = {"source": "genefer's proof / server / check modes (oracle/_ref/genefer_harness)", "cases": {}}
    for name, b, n, depth, seed in CASES:
        d = tempfile.mkdtemp()
        r = subprocess.run([HARNESS, d, str(b), str(n), str(depth), str(seed)], capture_output=True, text=True,
                           check=True)
        rnd = [int(x) for x in r.stdout.strip().splitlines()[-1].split()[1:]]
        lines = open(os.path.join(d, "results.txt")).read().strip().splitlines()
        assert len(lines) == 3, lines
        proof_keys, server_keys, check_keys = (dict(KEY.findall(ln)) for ln in lines)
        assert proof_keys["pkey"] == server_keys["pkey"] and server_keys["ckey"] == check_keys["ckey"]
        dst = os.path.join(HERE, "proof", name)
        os.makedirs(dst, exist_ok=True)
        shutil.copy(os.path.join(d, "g.proof"), os.path.join(dst, "g.proof"))
        shutil.copy(os.path.join(d, "g.cert"), os.path.join(dst, "g.cert"))
        shutil.rmtree(d)
        out["cases"][name] = {"b": b, "n": n, "depth": depth, "rnd": rnd, "res64": server_keys["res64"],
                              "old64": server_keys["old64"], "isPrp": "probable prime" in lines[1],
                              "pkey": server_keys["pkey"], "ckey": server_keys["ckey"]}
        print(name, out["cases"][name], flush=True)
    with open(os.path.join(HERE, "proof", "keys.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
