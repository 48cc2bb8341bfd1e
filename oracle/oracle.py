"""ctypes front-ends for the CPU oracle (test infrastructure only).

* ``Oracle``     - the plain-C restatement of the search path (erq_oracle.c),
                   built into oracle/_build/liberq_oracle.so.
* ``Reference``  - the reference's own search code (inc/ headers, compiled with
                   the shim) behind oracle/ref_harness.cpp, built into
                   oracle/_ref/liberq_ref.so (strict IEEE flags) and
                   oracle/_ref/liberq_ref_stock.so (the reference's -Ofast flags).

Only tests, __graft_entry__.smoke() and bench.py's CPU baseline use this
module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liberq_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "liberq_ref.so")
REF_STOCK_SO = os.path.join(HERE, "_ref", "liberq_ref_stock.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i16p = np.ctypeslib.ndpointer(np.int16, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


def build_oracle() -> str:
    """Compile the C restatement if it is missing (gcc only, a few seconds)."""
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return ORACLE_SO


def reference_available(stock: bool = False) -> bool:
    return os.path.exists(REF_STOCK_SO if stock else REF_SO)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Oracle:
    """The C restatement of IVF load + search (erq_oracle.h)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(build_oracle())
            lib.orc_index_load.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
            lib.orc_index_load.restype = C.c_int
            lib.orc_index_free.argtypes = [C.c_void_p]
            lib.orc_index_info.argtypes = [C.c_void_p, _u64p]
            lib.orc_centroids.argtypes = [C.c_void_p]
            lib.orc_centroids.restype = C.POINTER(C.c_float)
            lib.orc_rotation.argtypes = [C.c_void_p]
            lib.orc_rotation.restype = C.POINTER(C.c_float)
            lib.orc_cluster_sizes.argtypes = [C.c_void_p]
            lib.orc_cluster_sizes.restype = C.POINTER(C.c_uint64)
            lib.orc_long_code.argtypes = [C.c_void_p, C.c_uint64]
            lib.orc_long_code.restype = C.POINTER(C.c_uint8)
            lib.orc_l2sqr16.argtypes = [_f32p, _f32p, C.c_uint64]
            lib.orc_l2sqr16.restype = C.c_float
            lib.orc_probe.argtypes = [C.c_void_p, _f32p, C.c_uint64, _u32p, _f32p]
            lib.orc_prepare.argtypes = [C.c_uint64, _f32p, _f32p, C.c_float, _f32p, _i16p,
                                        C.POINTER(C.c_float), C.POINTER(C.c_float), _i32p]
            lib.orc_block_sums.argtypes = [C.c_uint64, _u8p, _i32p, _i32p]
            lib.orc_scan_cluster.argtypes = [C.c_void_p, _f32p, C.c_uint32, C.c_float, C.c_float,
                                             _i32p, _f32p, _u32p]
            lib.orc_scan_cluster.restype = C.c_uint64
            lib.orc_ex_decode.argtypes = [C.c_uint64, C.c_uint64, _u8p, _u8p]
            lib.orc_ex_ip.argtypes = [C.c_uint64, C.c_uint64, _f32p, _u8p]
            lib.orc_ex_ip.restype = C.c_float
            lib.orc_search.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64, _u32p, _f32p]
            lib.orc_search_batch.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64,
                                             C.c_uint64, _u32p, _f32p, C.c_int]
            lib.orc_trace.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64, C.c_uint64,
                                      _u32p, _f32p]
            lib.orc_trace.restype = C.c_uint64
            cls._lib = lib
        return cls._lib

    def __init__(self, path: str):
        h = C.c_void_p()
        rc = self.lib().orc_index_load(os.fsencode(path), C.byref(h))
        if rc != 0:
            raise OSError(f"orc_index_load({path}) failed with code {rc}")
        self.h = h
        info = np.zeros(5, np.uint64)
        self.lib().orc_index_info(self.h, info)
        self.N, self.DIM, self.D, self.K, self.EX = (int(x) for x in info)

    def close(self):
        if getattr(self, "h", None):
            self.lib().orc_index_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # raw views
    def centroids(self):
        p = self.lib().orc_centroids(self.h)
        return np.ctypeslib.as_array(p, shape=(self.K, self.D)).copy()

    def rotation(self):
        p = self.lib().orc_rotation(self.h)
        return np.ctypeslib.as_array(p, shape=(self.D, self.D)).copy()

    def cluster_sizes(self):
        p = self.lib().orc_cluster_sizes(self.h)
        return np.ctypeslib.as_array(p, shape=(self.K,)).copy()

    def long_code(self, pos: int):
        n = self.D * self.EX // 8
        p = self.lib().orc_long_code(self.h, pos)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    # stages
    def probe(self, q, nprobe):
        cids = np.zeros(nprobe, np.uint32)
        sq = np.zeros(nprobe, np.float32)
        self.lib().orc_probe(self.h, _f32(q), nprobe, cids, sq)
        return cids, sq

    def prepare(self, q, c, sqr_y):
        D = self.D
        unit_q = np.zeros(D, np.float32)
        qq = np.zeros(D, np.int16)
        lut = np.zeros(4 * D, np.int32)
        delta, sumq = C.c_float(), C.c_float()
        self.lib().orc_prepare(D, _f32(q), _f32(c), sqr_y, unit_q, qq, C.byref(delta),
                               C.byref(sumq), lut)
        return dict(unit_q=unit_q, qq=qq, delta=np.float32(delta.value),
                    sumq=np.float32(sumq.value), lut=lut)

    def scan_cluster(self, q, cid, sqr_y, distk):
        nb = (int(self.cluster_sizes()[cid]) + 31) // 32
        S = np.zeros(32 * max(nb, 1), np.int32)
        ipq = np.zeros(32 * max(nb, 1), np.float32)
        masks = np.zeros(max(nb, 1), np.uint32)
        n = self.lib().orc_scan_cluster(self.h, _f32(q), cid, sqr_y, distk, S, ipq, masks)
        return S[:32 * n], ipq[:32 * n], masks[:n]

    def ex_ip(self, unit_q, pos):
        code = self.long_code(pos)
        return np.float32(self.lib().orc_ex_ip(self.D, self.EX, _f32(unit_q), code))

    def ex_decode(self, code):
        out = np.zeros(self.D, np.uint8)
        self.lib().orc_ex_decode(self.D, self.EX, np.ascontiguousarray(code, np.uint8), out)
        return out

    def search(self, q, k, nprobe, nthreads=1):
        q = _f32(q).reshape(-1, self.D)
        nq = q.shape[0]
        ids = np.zeros((nq, k), np.uint32)
        d = np.zeros((nq, k), np.float32)
        self.lib().orc_search_batch(self.h, q, nq, k, nprobe, ids, d, nthreads)
        return ids, d

    def trace(self, q, k, nprobe, cap=1 << 20):
        ids = np.zeros(cap, np.uint32)
        d = np.zeros(cap, np.float32)
        n = self.lib().orc_trace(self.h, _f32(q), k, nprobe, cap, ids, d)
        return ids[:min(n, cap)], d[:min(n, cap)]


class Reference:
    """The reference's own search (oracle/ref_harness.cpp)."""

    _libs: dict = {}

    @classmethod
    def lib(cls, stock: bool = False):
        path = REF_STOCK_SO if stock else REF_SO
        if path not in cls._libs:
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} is not built (make -C oracle ref)")
            lib = C.CDLL(path)
            lib.ref_load.argtypes = [C.c_char_p]
            lib.ref_load.restype = C.c_void_p
            lib.ref_free.argtypes = [C.c_void_p]
            lib.ref_info.argtypes = [C.c_void_p, _u64p]
            lib.ref_search.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64, C.c_uint64,
                                       _u32p, C.c_int]
            lib.ref_search_timed.argtypes = lib.ref_search.argtypes
            lib.ref_search_timed.restype = C.c_double
            lib.ref_search_dists.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64,
                                             C.c_uint64, _u32p, _f32p]
            lib.ref_trace.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64, C.c_uint64,
                                      _u32p, _f32p]
            lib.ref_trace.restype = C.c_uint64
            lib.ref_probe.argtypes = [C.c_void_p, _f32p, C.c_uint64, _u32p, _f32p]
            lib.ref_centroid_dists.argtypes = [C.c_void_p, _f32p, _f32p]
            lib.ref_prepare.argtypes = [C.c_void_p, _f32p, C.c_uint32, C.c_float, _f32p, _i16p,
                                        C.POINTER(C.c_float), C.POINTER(C.c_float),
                                        C.POINTER(C.c_int32), _u8p]
            lib.ref_scan_cluster.argtypes = [C.c_void_p, _f32p, C.c_uint32, C.c_float,
                                             C.c_float, _f32p, _u32p]
            lib.ref_scan_cluster.restype = C.c_uint64
            lib.ref_ex_ip.argtypes = [C.c_void_p, _f32p, C.c_uint64]
            lib.ref_ex_ip.restype = C.c_float
            lib.ref_rotate.argtypes = [C.c_void_p, _f32p, C.c_uint64, _f32p]
            lib.ref_l2sqr16.argtypes = [_f32p, _f32p, C.c_uint64]
            lib.ref_l2sqr16.restype = C.c_float
            lib.ref_max_threads.restype = C.c_int
            cls._libs[path] = lib
        return cls._libs[path]

    def __init__(self, path: str, stock: bool = False):
        self.L = self.lib(stock)
        h = self.L.ref_load(os.fsencode(path))
        if not h:
            raise OSError(f"reference IVF::load({path}) failed")
        self.h = h
        info = np.zeros(5, np.uint64)
        self.L.ref_info(self.h, info)
        self.N, self.DIM, self.D, self.K, self.EX = (int(x) for x in info)

    def close(self):
        if getattr(self, "h", None):
            self.L.ref_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def search(self, q, k, nprobe, nthreads=1):
        q = _f32(q).reshape(-1, self.D)
        ids = np.zeros((q.shape[0], k), np.uint32)
        self.L.ref_search(self.h, q, q.shape[0], k, nprobe, ids, nthreads)
        return ids

    def search_timed(self, q, k, nprobe, nthreads=1):
        q = _f32(q).reshape(-1, self.D)
        ids = np.zeros((q.shape[0], k), np.uint32)
        sec = self.L.ref_search_timed(self.h, q, q.shape[0], k, nprobe, ids, nthreads)
        return ids, sec

    def search_dists(self, q, k, nprobe):
        q = _f32(q).reshape(-1, self.D)
        ids = np.zeros((q.shape[0], k), np.uint32)
        d = np.zeros((q.shape[0], k), np.float32)
        self.L.ref_search_dists(self.h, q, q.shape[0], k, nprobe, ids, d)
        return ids, d

    def trace(self, q, k, nprobe, cap=1 << 20):
        ids = np.zeros(cap, np.uint32)
        d = np.zeros(cap, np.float32)
        n = self.L.ref_trace(self.h, _f32(q), k, nprobe, cap, ids, d)
        return ids[:min(n, cap)], d[:min(n, cap)]

    def probe(self, q, nprobe):
        cids = np.zeros(nprobe, np.uint32)
        sq = np.zeros(nprobe, np.float32)
        self.L.ref_probe(self.h, _f32(q), nprobe, cids, sq)
        return cids, sq

    def centroid_dists(self, q):
        out = np.zeros(self.K, np.float32)
        self.L.ref_centroid_dists(self.h, _f32(q), out)
        return out

    def prepare(self, q, cid, sqr_y):
        D = self.D
        unit_q = np.zeros(D, np.float32)
        qq = np.zeros(D, np.int16)
        lut = np.zeros(8 * D, np.uint8)
        delta, sumq, shift = C.c_float(), C.c_float(), C.c_int32()
        self.L.ref_prepare(self.h, _f32(q), cid, sqr_y, unit_q, qq, C.byref(delta),
                           C.byref(sumq), C.byref(shift), lut)
        return dict(unit_q=unit_q, qq=qq, delta=np.float32(delta.value),
                    sumq=np.float32(sumq.value), shift=int(shift.value), lut=lut)

    def scan_cluster(self, q, cid, sqr_y, distk, nblocks):
        ipq = np.zeros(32 * max(nblocks, 1), np.float32)
        masks = np.zeros(max(nblocks, 1), np.uint32)
        n = self.L.ref_scan_cluster(self.h, _f32(q), cid, sqr_y, distk, ipq, masks)
        return ipq[:32 * n], masks[:n]

    def ex_ip(self, unit_q, pos):
        return np.float32(self.L.ref_ex_ip(self.h, _f32(unit_q), pos))

    def rotate(self, q):
        q = _f32(q).reshape(-1, self.DIM)
        out = np.zeros((q.shape[0], self.D), np.float32)
        self.L.ref_rotate(self.h, q, q.shape[0], out)
        return out

    @classmethod
    def max_threads(cls, stock: bool = False):
        return int(cls.lib(stock).ref_max_threads())


REF_LOWACC_SO = os.path.join(HERE, "_ref", "liberq_ref_lowacc.so")


class LowAccReference:
    """The reference's non-HIGH_ACC format and Searcher (oracle/ref_lowacc.cpp):
    builds indexes with IVF::construct + save and searches them with the
    reference's own Searcher (inc/index/Searcher.hpp)."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_LOWACC_SO)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_LOWACC_SO):
                raise FileNotFoundError(f"{REF_LOWACC_SO} is not built (make -C oracle ref)")
            lib = C.CDLL(REF_LOWACC_SO)
            lib.lref_build.argtypes = [_f32p, C.c_uint64, C.c_uint64, _f32p, C.c_uint64, _u32p,
                                       C.c_uint64, C.c_char_p]
            lib.lref_build.restype = C.c_int
            lib.lref_load.argtypes = [C.c_char_p]
            lib.lref_load.restype = C.c_void_p
            lib.lref_free.argtypes = [C.c_void_p]
            lib.lref_info.argtypes = [C.c_void_p, _u64p]
            lib.lref_rotate.argtypes = [C.c_void_p, _f32p, C.c_uint64, _f32p]
            lib.lref_search_dists.argtypes = [C.c_void_p, _f32p, C.c_uint64, C.c_uint64,
                                              C.c_uint64, _u32p, _f32p]
            cls._lib = lib
        return cls._lib

    @classmethod
    def build(cls, data, centroids, cluster_ids, bits: int, path: str) -> None:
        """IVF(n, dim, K, bits).construct(data, centroids, cluster_ids).save(path)."""
        x = _f32(data)
        c = _f32(centroids)
        ids = np.ascontiguousarray(cluster_ids, dtype=np.uint32)
        rc = cls.lib().lref_build(x, x.shape[0], x.shape[1], c, c.shape[0], ids, bits,
                                  os.fsencode(path))
        if rc != 0:
            raise RuntimeError("lref_build failed")

    def __init__(self, path: str):
        h = self.lib().lref_load(os.fsencode(path))
        if not h:
            raise OSError(f"reference IVF::load({path}) failed")
        self.h = h
        info = np.zeros(5, np.uint64)
        self.lib().lref_info(self.h, info)
        self.N, self.DIM, self.D, self.K, self.EX = (int(x) for x in info)

    def close(self):
        if getattr(self, "h", None):
            self.lib().lref_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def rotate(self, q):
        q = _f32(q).reshape(-1, self.DIM)
        out = np.zeros((q.shape[0], self.D), np.float32)
        self.lib().lref_rotate(self.h, q, q.shape[0], out)
        return out

    def search_dists(self, q, k, nprobe):
        q = _f32(q).reshape(-1, self.D)
        ids = np.zeros((q.shape[0], k), np.uint32)
        d = np.zeros((q.shape[0], k), np.float32)
        self.lib().lref_search_dists(self.h, q, q.shape[0], k, nprobe, ids, d)
        return ids, d
