"""genefer22_b200: B200-native modular-squaring engine for generalized Fermat
PRP tests b^(2^n) + 1, behind genefer's `transform` interface.

The engine is libgfcuda.so (CUDA kernels for sm_100a + C ABI,
include/gfcuda.h).  This package is its Python host side: the transform
mirror (``Transform``, ``Batch``), genefer's residue utilities (``gint``) and
the PRP / Gerbicz-Li driver (``genefer``).
"""
from ._lib import GfcError, lib, lib_path
from .transform import Batch, Graph, Transform

__all__ = ["Batch", "Graph", "Transform", "GfcError", "lib", "lib_path"]
