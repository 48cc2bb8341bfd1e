"""IVF clustering on the GPU (include/erq.h, erq_kmeans*): the step the
reference runs offline with faiss (python/ivf.py:5-34) to produce the
centroid and cluster-id files that create_index reads."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, load_library


def _ptr(a):
    return C.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)


def kmeans(data, k: int, iters: int = 20, seed: int = 0, device: int = 0):
    """Returns (centroids float32 [k, dim], assign uint32 [n]) as numpy arrays.
    ``data`` may be a numpy array or a torch tensor (host or device)."""
    if not hasattr(data, "data_ptr"):
        data = np.ascontiguousarray(data, np.float32)
    n, dim = data.shape
    cent = np.empty((k, dim), np.float32)
    assign = np.empty(n, np.uint32)
    check(load_library().erq_kmeans(_ptr(data), n, dim, k, iters, seed, _ptr(cent), _ptr(assign),
                                    device))
    return cent, assign


def kmeans_step(data, centroids, seed: int = 0, device: int = 0):
    """One Lloyd iteration from ``centroids``: (new centroids, assign, counts)."""
    data = np.ascontiguousarray(data, np.float32)
    c = np.ascontiguousarray(centroids, np.float32)
    n, dim = data.shape
    k = c.shape[0]
    out = np.empty_like(c)
    assign = np.empty(n, np.uint32)
    counts = np.empty(k, np.uint32)
    check(load_library().erq_kmeans_step(_ptr(data), n, dim, k, _ptr(c), seed, _ptr(out),
                                         _ptr(assign), _ptr(counts), device))
    return out, assign, counts
