"""genefer22_b200: B200-native modular-squaring engine for generalized Fermat
PRP tests b^(2^n) + 1, behind genefer's `transform` interface.

The engine is libgfcuda.so (CUDA kernels for sm_100a + C ABI,
include/gfcuda.h).  This package is its Python host side:

* ``transform``: the transform mirror (``Transform``, ``Batch``, ``Graph``)
* ``gint``, ``exponent``: genefer's residue utilities and the exponent
* ``genefer``: the PRP / Gerbicz-Li driver, one test or a batch
* ``verify``: periodic Gerbicz-Li verification with rollback
* ``autotune``, ``mixed``: plan choice per size class, uneven batches
* ``serve``: the continuous-batching request loop
* ``shard``: test queues over GPUs
* ``proof``, ``prime``: proof / server / check modes, file formats and
  contexts, the deterministic test
"""
from ._lib import GfcError, lib, lib_path
from .transform import Batch, Graph, Transform

__all__ = ["Batch", "Graph", "Transform", "GfcError", "lib", "lib_path"]
