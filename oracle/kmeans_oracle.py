"""CPU restatement of one k-means iteration of the library (test
infrastructure only): the clustering step of the reference's pipeline
(python/ivf.py:5-34, faiss IVF training) as the library runs it -
assignment to the nearest centroid (ties to the smaller index), means in
float64, empty clusters split from a populated one chosen with probability
proportional to (size - 1), c * (1 +- 1/1024) alternately per dimension,
with splitmix64 as the random stream."""
from __future__ import annotations

import numpy as np

MASK = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea and Flood, 2014)."""

    def __init__(self, seed: int):
        self.s = seed & MASK

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def init_rows(n: int, k: int, seed: int) -> np.ndarray:
    """The k distinct rows the library starts from (partial Fisher-Yates)."""
    rng = SplitMix64(seed)
    perm = np.arange(n, dtype=np.int64)
    for i in range(k):
        j = i + rng.next() % (n - i)
        perm[i], perm[j] = perm[j], perm[i]
    return perm[:k].copy()


def exact_dists(x: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Squared L2 distances in float64 [n, k]."""
    x = x.astype(np.float64)
    c = c.astype(np.float64)
    return (x * x).sum(1)[:, None] + (c * c).sum(1)[None, :] - 2.0 * x @ c.T


def update(x: np.ndarray, assign: np.ndarray, c_in: np.ndarray, seed: int):
    """Means of the given assignment, then the empty-cluster splits.
    Returns (centroids float32 [k, dim], counts [k])."""
    k, dim = c_in.shape
    cnt = np.bincount(assign, minlength=k)
    sums = np.zeros((k, dim))
    np.add.at(sums, assign, x.astype(np.float64))
    c = c_in.astype(np.float32).copy()
    nz = cnt > 0
    c[nz] = (sums[nz] / cnt[nz, None]).astype(np.float32)
    rng = SplitMix64(seed)
    cf = cnt.astype(np.float64)
    sign = np.where(np.arange(dim) % 2 == 0, 1.0, -1.0).astype(np.float32)
    eps = np.float32(1.0 / 1024.0)
    for ci in range(k):
        if cf[ci] != 0:
            continue
        w = np.maximum(cf - 1.0, 0.0)
        total = w.sum()
        if total > 0:
            u = rng.uniform() * total
            run, cj = 0.0, 0
            for cj in range(k - 1):
                run += w[cj]
                if u < run:
                    break
            else:
                cj = k - 1
        else:
            cj = int(np.argmax(cf))
        v = c[cj].copy()
        c[ci] = v * (np.float32(1) + eps * sign)
        c[cj] = v * (np.float32(1) - eps * sign)
        cf[ci] = np.floor(cf[cj] / 2)
        cf[cj] -= cf[ci]
    return c, cnt
