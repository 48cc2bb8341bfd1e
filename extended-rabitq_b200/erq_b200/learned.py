"""Learned probing: per-query probe depth predicted by a small MLP.

Labels come from the plain search itself: for a query, the label is the
smallest class c whose probe count bins[c] gives the same top-k set as the
deepest class bins[-1] (the depth at which the plain method's result stops
changing, measured on the class grid).  The deepest class stands in for
exhaustive probing; ``exhaustive_agreement`` measures how often its top-k
already is the exhaustive one.  ``scaled_bins`` spreads the classes
geometrically up to twice the workload's fixed nprobe.  The MLP (trained on the GPU by the
library's own forward/backward kernels) maps a query's features (a sketch of
the rotated query and its 64 nearest exact centroid distances) to a
distribution over the classes; the learned search scans the smallest depth
whose cumulative probability reaches a confidence level, or the fixed
nprobe when the model is unsure.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import check, load_library

DEFAULT_BINS = (1, 2, 3, 4, 6, 8, 12, 16)
N_FEATURES = 320
N_BINS = 8
N_PARAMS = 150024


def scaled_bins(nprobe: int, K: int) -> tuple:
    """The 8 probe depths of a workload whose fixed nprobe is `nprobe`: up to
    twice nprobe (at least 16, at most K), geometric from 1/64 of the top, so
    that a model can both cut and deepen the fixed search.  DEFAULT_BINS when
    the top is 16 or less."""
    top = min(K, max(16, 2 * nprobe))
    if top <= 16:
        return tuple(min(b, K) for b in DEFAULT_BINS)
    lo = max(1.0, top / 64.0)
    r = (top / lo) ** (1.0 / (N_BINS - 1))
    bins = []
    for i in range(N_BINS):
        b = int(round(lo * r ** i))
        b = max(b, bins[-1] + 1 if bins else 1)
        bins.append(b)
    bins[-1] = top
    for i in range(N_BINS - 2, -1, -1):  # strictly increasing below the top
        bins[i] = min(bins[i], bins[i + 1] - 1)
    return tuple(bins)


def exhaustive_agreement(ivf, rotated_queries, k: int, depth: int) -> float:
    """Fraction of queries whose top-k set at `depth` probes equals the
    top-k set of the exhaustive search (every cluster probed): how well the
    deepest label bin stands in for exhaustive probing."""
    q = np.ascontiguousarray(rotated_queries, np.float32).reshape(-1, ivf.D)
    a, _ = ivf.search_batch(q, k, min(depth, ivf.K), with_dists=False)
    b, _ = ivf.search_batch(q, k, ivf.K, with_dists=False)
    return float(np.all(np.sort(a, 1) == np.sort(b, 1), axis=1).mean())


def fallback_rate(model, features, min_prob: float) -> float:
    """Fraction of queries whose most likely depth has probability below
    min_prob, which the learned search sends to the fixed nprobe."""
    if min_prob <= 0:
        return 0.0
    p = model.predict(features)
    return float((p.max(axis=1) < min_prob).mean())


def probe_features(ivf, rotated_queries) -> np.ndarray:
    q = np.ascontiguousarray(rotated_queries, np.float32).reshape(-1, ivf.D)
    out = np.empty((q.shape[0], N_FEATURES), np.float32)
    check(load_library().erq_probe_features(ivf._h, q.ctypes.data, q.shape[0],
                                            out.ctypes.data, None))
    return out


def make_labels(ivf, rotated_queries, k: int, bins=DEFAULT_BINS) -> np.ndarray:
    """Smallest class whose depth already returns the deepest class's top-k set."""
    q = np.ascontiguousarray(rotated_queries, np.float32).reshape(-1, ivf.D)
    bins = [min(b, ivf.K) for b in bins]
    results = []
    for b in bins:
        ids, _ = ivf.search_batch(q, k, b, with_dists=False)
        results.append(np.sort(ids, axis=1))
    final = results[-1]
    labels = np.full(q.shape[0], len(bins) - 1, np.uint8)
    for c in range(len(bins) - 2, -1, -1):
        same = np.all(results[c] == final, axis=1)
        labels[same] = c
    return labels


class ProbeModel:
    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self._lib = load_library()

    @classmethod
    def train(cls, features, labels, bins=DEFAULT_BINS, epochs: int = 10, batch: int = 1024,
              lr: float = 1e-3, seed: int = 0, device: int = 0):
        f = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(labels, np.uint8)
        b = np.ascontiguousarray(bins, np.uint32)
        if f.shape[1] != N_FEATURES or b.size != N_BINS or y.shape[0] != f.shape[0]:
            raise ValueError("features [n, 320], labels [n], 8 bins expected")
        h = C.c_void_p()
        loss = C.c_float()
        check(load_library().erq_probe_model_train(f.ctypes.data, y.ctypes.data, f.shape[0],
                                                   b.ctypes.data, epochs, batch, lr, seed,
                                                   device, C.byref(h), C.byref(loss)))
        m = cls(h)
        m.final_loss = float(loss.value)
        return m

    @classmethod
    def load(cls, path, device: int = 0):
        h = C.c_void_p()
        check(load_library().erq_probe_model_load(os.fsencode(os.fspath(path)), device,
                                                  C.byref(h)))
        return cls(h)

    def save(self, path) -> None:
        check(self._lib.erq_probe_model_save(self._h, os.fsencode(os.fspath(path))))

    def free(self) -> None:
        if self._h:
            self._lib.erq_probe_model_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def predict(self, features) -> np.ndarray:
        f = np.ascontiguousarray(features, np.float32)
        out = np.empty((f.shape[0], N_BINS), np.float32)
        check(self._lib.erq_probe_model_predict(self._h, f.ctypes.data, f.shape[0],
                                                out.ctypes.data, None))
        return out

    def params(self):
        p = np.empty(N_PARAMS, np.float32)
        mean = np.empty(N_FEATURES, np.float32)
        std = np.empty(N_FEATURES, np.float32)
        bins = np.empty(N_BINS, np.uint32)
        check(self._lib.erq_debug_probe_model_params(self._h, p.ctypes.data, mean.ctypes.data,
                                                     std.ctypes.data, bins.ctypes.data))
        return p, mean, std, bins

    def grads(self, features, labels):
        f = np.ascontiguousarray(features, np.float32)
        y = np.ascontiguousarray(labels, np.uint8)
        g = np.empty(N_PARAMS, np.float32)
        loss = C.c_float()
        check(self._lib.erq_debug_probe_model_grads(self._h, f.ctypes.data, y.ctypes.data,
                                                    f.shape[0], C.byref(loss), g.ctypes.data))
        return float(loss.value), g


def search_learned(ivf, model: ProbeModel, rotated_queries, k: int, nprobe_fallback: int,
                   confidence: float = 0.9, min_prob: float = 0.0, stream=None):
    """Returns (ids, dists, nprobe_used); numpy host buffers."""
    q = np.ascontiguousarray(rotated_queries, np.float32).reshape(-1, ivf.D)
    nq = q.shape[0]
    ids = np.empty((nq, k), np.uint32)
    d = np.empty((nq, k), np.float32)
    used = np.empty(nq, np.uint32)
    st = None if stream is None else C.c_void_p(stream.cuda_stream)
    check(load_library().erq_search_learned(ivf._h, model._h, q.ctypes.data, nq, k,
                                            nprobe_fallback, confidence, min_prob, ids.ctypes.data,
                                            d.ctypes.data, used.ctypes.data, st))
    return ids, d, used


def search_learned_buffers(ivf, model: ProbeModel, queries, k: int, nprobe_fallback: int,
                           confidence: float, ids, dists, used=None, raw: bool = True,
                           min_prob: float = 0.0, stream=None) -> None:
    """Learned search into caller buffers (numpy arrays or torch tensors, host
    or device): raw DIM-float queries when `raw`, else rotated ones."""
    ptr = lambda t: None if t is None else C.c_void_p(  # noqa: E731
        t.data_ptr() if hasattr(t, "data_ptr") else t.ctypes.data)
    fn = load_library().erq_search_learned_raw if raw else load_library().erq_search_learned
    st = None if stream is None else C.c_void_p(stream.cuda_stream)
    check(fn(ivf._h, model._h, ptr(queries), int(queries.shape[0]), k, nprobe_fallback,
             confidence, min_prob, ptr(ids), ptr(dists), ptr(used), st))
