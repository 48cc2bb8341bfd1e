"""Batched search plans (include/erq.h, erq_plan_*).

A plan owns the device buffers for batches of up to ``max_batch`` queries,
captures the search of each batch size into a CUDA graph on first use and
replays it, and scans over a (cluster x query block x cluster chunk) work list
whose tile shape ``autotune`` picks per batch size.  Results equal
``IVF.search_batch`` (no model) or ``learned.search_learned`` (with a model).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import PlanTuning, check, load_library


def _ptr(a):
    if a is None:
        return None
    return C.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data)


class Plan:
    def __init__(self, ivf, max_batch: int, k: int, nprobe: int, model=None, raw: bool = False):
        self.ivf, self.k, self.nprobe, self.max_batch, self.raw = ivf, k, nprobe, max_batch, raw
        self.model = model
        self._lib = load_library()
        h = C.c_void_p()
        check(self._lib.erq_plan_create(ivf._h, model._h if model is not None else None, max_batch,
                                        k, nprobe, 1 if raw else 0, C.byref(h)))
        self._h = h

    @property
    def cols(self) -> int:
        return self.ivf.DIM if self.raw else self.ivf.D

    def free(self) -> None:
        if self._h:
            self._lib.erq_plan_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def set_learned(self, confidence: float, min_prob: float = 0.0) -> None:
        check(self._lib.erq_plan_set_learned(self._h, confidence, min_prob))

    def autotune(self, sample, reps: int = 3):
        q = np.ascontiguousarray(sample, np.float32).reshape(-1, self.cols)
        t = PlanTuning()
        ms = C.c_float()
        check(self._lib.erq_plan_autotune(self._h, _ptr(q), q.shape[0], reps, C.byref(t),
                                          C.byref(ms)))
        return t.as_dict(), float(ms.value)

    def set_tuning(self, batch: int, queries_per_item: int, blocks_per_item: int, warps: int,
                   refine_warps: int = 0) -> None:
        """refine_warps: 4, 32 (wide refinement form) or 0 (by batch size)."""
        t = PlanTuning(queries_per_item, blocks_per_item, warps, refine_warps)
        check(self._lib.erq_plan_set_tuning(self._h, batch, C.byref(t)))

    def tuning(self, batch: int) -> dict:
        t = PlanTuning()
        check(self._lib.erq_plan_get_tuning(self._h, batch, C.byref(t)))
        return t.as_dict()

    def set_graphs(self, on: bool) -> None:
        check(self._lib.erq_plan_set_graphs(self._h, 1 if on else 0))

    def set_pipeline(self, chunks: int) -> None:
        """Pieces a host-buffer batch runs as (1: one piece, 0: by batch size)."""
        check(self._lib.erq_plan_set_pipeline(self._h, chunks))

    def search_buffers_async(self, queries, ids, dists=None, nprobe_used=None, stream=None) -> None:
        """search_buffers without waiting (erq_plan_search_async): results are
        valid once ``stream`` is synchronised; host buffers should be pinned."""
        st = None if stream is None else C.c_void_p(stream.cuda_stream)
        check(self._lib.erq_plan_search_async(self._h, _ptr(queries), int(queries.shape[0]),
                                              _ptr(ids), _ptr(dists), _ptr(nprobe_used), st))

    def device_bytes(self) -> int:
        return int(self._lib.erq_plan_device_bytes(self._h))

    def search(self, queries, with_dists: bool = True, with_nprobe: bool = False):
        """numpy in, numpy out: (ids, dists or None, nprobe_used or None)."""
        q = np.ascontiguousarray(queries, np.float32).reshape(-1, self.cols)
        nq = q.shape[0]
        ids = np.empty((nq, self.k), np.uint32)
        d = np.empty((nq, self.k), np.float32) if with_dists else None
        u = np.empty(nq, np.uint32) if with_nprobe else None
        check(self._lib.erq_plan_search(self._h, _ptr(q), nq, _ptr(ids), _ptr(d), _ptr(u), None))
        return ids, d, u

    def search_buffers(self, queries, ids, dists=None, nprobe_used=None, stream=None) -> None:
        """Caller buffers (numpy arrays or torch tensors, host or device)."""
        st = None if stream is None else C.c_void_p(stream.cuda_stream)
        check(self._lib.erq_plan_search(self._h, _ptr(queries), int(queries.shape[0]), _ptr(ids),
                                        _ptr(dists), _ptr(nprobe_used), st))
