"""Reader / writer of the reference's index file (IVF::save / IVF::load,
inc/index/IVF.hpp:219-293), HIGH_ACC_FAST_SCAN block layout.

Little-endian, no magic or version:
  N, DIM, K, EX_BITS           4 x uint64
  cluster_sizes                K x uint64 (sum = N)
  rotation P                   D x D float32, row-major (inc/index/Rotator.hpp:34-55)
  rotated centroids            K x D float32 (FlatInitializer, K < 20000)
  short data                   sum_c ceil(n_c/32) blocks of 4D code bytes + 32 float32
  long (EX-bit) codes          N x D*EX/8 bytes
  EX factors (xipnorm)         N x float32
  ids                          N x uint32
Clusters are stored contiguously in cluster order.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np


@dataclasses.dataclass
class IndexArrays:
    N: int
    DIM: int
    K: int
    EX: int
    sizes: np.ndarray        # [K] uint64
    P: np.ndarray            # [D, D] float32
    centroids: np.ndarray    # [K, D] float32
    short: np.ndarray        # [blocks, 4D + 128] uint8
    long_code: np.ndarray    # [N, D*EX/8] uint8
    xipnorm: np.ndarray      # [N] float32
    ids: np.ndarray          # [N] uint32

    @property
    def D(self) -> int:
        return (self.DIM + 63) // 64 * 64

    def first_block(self) -> np.ndarray:
        nb = (self.sizes.astype(np.int64) + 31) // 32
        return np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)

    def first_vec(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.sizes.astype(np.int64))[:-1]]).astype(np.int64)


def read_index(path: str | os.PathLike, mmap: bool = True) -> IndexArrays:
    mm = np.memmap(path, dtype=np.uint8, mode="r") if mmap else np.fromfile(path, np.uint8)
    off = 0

    def take(dtype, count):
        nonlocal off
        nbytes = np.dtype(dtype).itemsize * count
        if off + nbytes > mm.size:
            raise ValueError(f"{path}: truncated")
        a = mm[off:off + nbytes].view(dtype)
        off += nbytes
        return a

    N, DIM, K, EX = (int(x) for x in take(np.uint64, 4))
    D = (DIM + 63) // 64 * 64
    sizes = np.array(take(np.uint64, K))
    if int(sizes.sum()) != N:
        raise ValueError(f"{path}: cluster sizes sum to {int(sizes.sum())}, N = {N}")
    P = take(np.float32, D * D).reshape(D, D)
    cent = take(np.float32, K * D).reshape(K, D)
    blocks = int(((sizes + 31) // 32).sum())
    short = take(np.uint8, blocks * (4 * D + 128)).reshape(blocks, 4 * D + 128)
    long_code = take(np.uint8, N * (D * EX // 8)).reshape(N, D * EX // 8)
    xip = take(np.float32, N)
    ids = take(np.uint32, N)
    return IndexArrays(N, DIM, K, EX, sizes, P, cent, short, long_code, xip, ids)


def write_index(path: str | os.PathLike, a: IndexArrays) -> None:
    with open(path, "wb") as f:
        np.array([a.N, a.DIM, a.K, a.EX], np.uint64).tofile(f)
        np.asarray(a.sizes, np.uint64).tofile(f)
        np.ascontiguousarray(a.P, np.float32).tofile(f)
        np.ascontiguousarray(a.centroids, np.float32).tofile(f)
        np.ascontiguousarray(a.short, np.uint8).tofile(f)
        np.ascontiguousarray(a.long_code, np.uint8).tofile(f)
        np.ascontiguousarray(a.xipnorm, np.float32).tofile(f)
        np.ascontiguousarray(a.ids, np.uint32).tofile(f)
