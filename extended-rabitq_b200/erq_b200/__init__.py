"""B200 IVF search for Extended-RaBitQ indexes.

The compute path is liberq.so (hand-written sm_100a CUDA behind the C ABI of
include/erq.h); this package is its Python host side:

* ``IVF``       - mirror of the reference's IVF class (load / search / rotate)
* ``vecs``      - .fvecs / .ivecs IO in the reference's file format
* ``datasets``  - seeded synthetic datasets, k-means, exact ground truth
* ``indexfile`` - reader/writer of the reference's index file format
* ``metrics``   - recall@k and the reference's average distance ratio
* ``plan``      - batched, graph-captured, autotuned search plans
* ``learned``   - learned probing (probe MLP)
* ``clustering`` - IVF clustering (k-means) on the GPU
"""
from ._lib import EXPORTED_SYMBOLS, ErqError, load_library  # noqa: F401
from .ivf import IVF  # noqa: F401
from .plan import Plan  # noqa: F401

__all__ = ["IVF", "Plan", "ErqError", "load_library", "EXPORTED_SYMBOLS"]
