"""Host-side mirror of the reference's IVF class (inc/index/IVF.hpp:62-127).

``IVF.load`` / ``IVF.search`` / ``IVF.padded_dim`` / ``IVF.k`` keep the
reference's names and argument meaning; the work happens in liberq.so on one
GPU.  Inputs may be numpy arrays (host memory) or torch tensors (host or
device memory); outputs follow the inputs' kind unless buffers are passed in.
Index construction (IVF(n, dim, k, b) + construct + save) is done by the
reference's create_index; this class reads what it writes.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import IndexInfo, check, load_library

try:  # torch is optional: numpy host buffers work without it
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_torch(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor)


def _ptr(x, dtype_np, dtype_torch_ok):
    """(pointer, keepalive) of a C-contiguous buffer of the given element type."""
    if _is_torch(x):
        if x.dtype not in dtype_torch_ok:
            raise TypeError(f"tensor dtype {x.dtype} not in {dtype_torch_ok}")
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(x.data_ptr()), x
    a = np.asarray(x)
    if a.dtype != dtype_np or not a.flags["C_CONTIGUOUS"]:
        raise TypeError(f"expected a C-contiguous {dtype_np} array, got {a.dtype}")
    return C.c_void_p(a.ctypes.data), a


def _stream_handle(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)  # torch.cuda.Stream


class IVF:
    """An Extended-RaBitQ IVF index resident on one GPU."""

    def __init__(self, path: str | os.PathLike | None = None, device: int = 0):
        self._h = C.c_void_p()
        self._lib = load_library()
        if path is not None:
            self.load(path, device)

    # -- IVF::load (inc/index/IVF.hpp:254-293)
    def load(self, path: str | os.PathLike, device: int = 0) -> None:
        self.free()
        h = C.c_void_p()
        check(self._lib.erq_index_load(os.fsencode(os.fspath(path)), int(device), C.byref(h)))
        self._h = h
        info = IndexInfo()
        check(self._lib.erq_index_get_info(self._h, C.byref(info)))
        self.N, self.DIM, self.D = int(info.n), int(info.dim), int(info.padded_dim)
        self.K, self.EX_BITS = int(info.num_clusters), int(info.ex_bits)
        self.device = int(info.device)
        self.device_bytes = int(info.device_bytes)
        self.block_factors = int(info.block_factors)

    def free(self) -> None:
        if self._h:
            self._lib.erq_index_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def _need(self):
        if not self._h:
            raise RuntimeError("index not loaded")

    # -- IVF::padded_dim / IVF::k (inc/index/IVF.hpp:86-90)
    def padded_dim(self) -> int:
        return self.D

    def k(self) -> int:
        return self.K

    # -- Rotator::rotate on DIM-float queries (inc/index/Rotator.hpp:60-63)
    def rotate(self, queries, out=None, stream=None):
        self._need()
        nq = int(queries.shape[0])
        if out is None:
            if _is_torch(queries):
                out = torch.empty((nq, self.D), dtype=torch.float32, device=queries.device)
            else:
                out = np.empty((nq, self.D), np.float32)
        qp, _k1 = _ptr(queries, np.float32, (torch.float32,) if torch else ())
        op, _k2 = _ptr(out, np.float32, (torch.float32,) if torch else ())
        check(self._lib.erq_rotate(self._h, qp, nq, op, _stream_handle(stream)))
        return out

    def _alloc_out(self, like, nq, k, want_dists):
        if _is_torch(like):
            ids = torch.empty((nq, k), dtype=torch.int32, device=like.device)
            d = torch.empty((nq, k), dtype=torch.float32, device=like.device) if want_dists else None
        else:
            ids = np.empty((nq, k), np.uint32)
            d = np.empty((nq, k), np.float32) if want_dists else None
        return ids, d

    def _search(self, fn, queries, k, nprobe, ids, dists, want_dists, stream):
        self._need()
        nq = int(queries.shape[0])
        if ids is None:
            ids, d_new = self._alloc_out(queries, nq, k, want_dists and dists is None)
            dists = dists if dists is not None else d_new
        elif dists is None and want_dists:
            _, dists = self._alloc_out(ids, nq, k, True)
        tf = (torch.float32,) if torch else ()
        ti = (torch.int32,) if torch else ()
        qp, _k1 = _ptr(queries, np.float32, tf)
        ip, _k2 = _ptr(ids, np.uint32, ti)
        dp, _k3 = (_ptr(dists, np.float32, tf) if dists is not None else (None, None))
        check(fn(self._h, qp, nq, int(k), int(nprobe), ip, dp, _stream_handle(stream)))
        return ids, dists

    def search_batch(self, rotated_queries, k: int, nprobe: int, ids=None, dists=None,
                     with_dists: bool = True, stream=None):
        """IVF::search for a batch of rotated queries [nq, D]; returns (ids, dists)."""
        return self._search(self._lib.erq_search, rotated_queries, k, nprobe, ids, dists,
                            with_dists, stream)

    def search_raw(self, queries, k: int, nprobe: int, ids=None, dists=None,
                   with_dists: bool = True, stream=None):
        """Rotate [nq, DIM] queries then search (test_search's sequence)."""
        return self._search(self._lib.erq_search_raw, queries, k, nprobe, ids, dists,
                            with_dists, stream)

    # -- IVF::search(query, data, k, nprobe, results) (inc/index/IVF.hpp:295-324)
    def search(self, query, data, k: int, nprobe: int, results) -> None:
        """One rotated query (D floats); ``data`` is unused, as in the reference."""
        del data
        q = np.ascontiguousarray(np.asarray(query, np.float32).reshape(1, self.D))
        ids, _ = self.search_batch(q, k, nprobe, with_dists=False)
        results[:k] = ids[0]

    # -- per-stage dumps (include/erq_debug.h)
    def debug_centroid_dists(self, rotated_queries):
        q = np.ascontiguousarray(rotated_queries, np.float32).reshape(-1, self.D)
        out = np.empty((q.shape[0], self.K), np.float32)
        check(self._lib.erq_debug_centroid_dists(self._h, q.ctypes.data, q.shape[0],
                                                 out.ctypes.data))
        return out

    def debug_probe(self, rotated_queries, nprobe: int):
        q = np.ascontiguousarray(rotated_queries, np.float32).reshape(-1, self.D)
        cids = np.empty((q.shape[0], nprobe), np.uint32)
        sq = np.empty((q.shape[0], nprobe), np.float32)
        check(self._lib.erq_debug_probe(self._h, q.ctypes.data, q.shape[0], nprobe,
                                        cids.ctypes.data, sq.ctypes.data))
        return cids, sq

    def debug_scan(self, rotated_queries, nprobe: int):
        q = np.ascontiguousarray(rotated_queries, np.float32).reshape(-1, self.D)
        nq = q.shape[0]
        cap = int(self._lib.erq_debug_scan_capacity(self._h, nq, nprobe))
        cids = np.empty((nq, nprobe), np.uint32)
        sq = np.empty((nq, nprobe), np.float32)
        delta = np.empty((nq, nprobe), np.float32)
        sumq = np.empty((nq, nprobe), np.float32)
        offs = np.empty((nq, nprobe), np.uint64)
        S = np.zeros(max(cap, 1), np.int32)
        check(self._lib.erq_debug_scan(self._h, q.ctypes.data, nq, nprobe, cids.ctypes.data,
                                       sq.ctypes.data, delta.ctypes.data, sumq.ctypes.data,
                                       offs.ctypes.data, S.ctypes.data, cap))
        return dict(cids=cids, sqr_y=sq, delta=delta, sumq=sumq, offsets=offs, S=S)
