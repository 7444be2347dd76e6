"""The C++ drop-in (include/transformCUDA.h) against genefer's own headers:
it compiles (CPU, when the genefer sources are present) and runs genefer's
quick-test sequence to the reference's known residues (GPU, prebuilt driver)."""
import os
import subprocess

import pytest

from ref_tree import genefer_tree

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_TREE = genefer_tree()              # GENEFER_REF, else oracle/Makefile's default
REFERENCE_SRC = os.path.join(_TREE, "src") if _TREE else ""
DRIVER = os.path.join(ROOT, "tests", "cpp", "_build", "kat_transformCUDA")

# src/main.cpp:417-425
KATS = {(33160956, 11): "9E2D51DA6C7C3F54", (23448336, 12): "81CFF004ACE85CAA", (2000000000, 12): "E5F3EA34F6C68EBD"}


@pytest.mark.skipif(not REFERENCE_SRC, reason="genefer sources not present")
def test_header_compiles_against_genefer():
    src = '#include "transform.h"\n#include "transformCUDA.h"\nint main() { return sizeof(transformCUDA) > 0 ? 0 : 1; }\n'
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-Wno-sign-conversion",
                        f"-I{REFERENCE_SRC}", f"-I{ROOT}/include", f"-I{ROOT}/oracle/gmp_standin", "-x", "c++", "-"],
                       input=src, text=True, capture_output=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DRIVER), reason="C++ driver not built (needs the genefer sources at build time)")
def test_transform_cuda_quick_kats():
    args = []
    for (b, n) in KATS:
        args += [str(b), str(n)]
    r = subprocess.run([DRIVER, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == len(KATS)
    for ln in lines:
        b, n, res64, is_prp, gl_ok, ctx_ok = ln.split()
        assert res64 == KATS[(int(b), int(n))]
        assert is_prp == "0" and gl_ok == "1" and ctx_ok == "1"
