"""Seeded synthetic datasets, IVF clustering and exact ground truth.

The reference is benchmarked on embedding datasets that are not available
here; these generators stand in for them with the same shapes and value
distributions:

* ``gaussian_mixture``: centres ~ N(0, I), isotropic within-component noise
  (the 100k x 128 small case: 256 centres, sigma 0.3).
* ``sphere_mixture``: centres uniform on the unit sphere, points are the
  centre plus tangent Gaussian noise, re-normalised to unit length (the
  1M x 1536 unit-norm embedding case, sigma 0.05), optionally with Zipf
  component weights (the uneven-cluster cases).

``kmeans`` replaces the reference's faiss clustering step (python/ivf.py:5-34)
and ``ground_truth`` its brute-force top-k (python/compute_gt.py:9-19), here in
float64.  numpy versions serve small cases; the ``*_torch`` versions run on a
GPU for the large ones.
"""
from __future__ import annotations

import numpy as np


def zipf_weights(n: int, s: float) -> np.ndarray:
    w = 1.0 / np.arange(1, n + 1, dtype=np.float64) ** s
    return w / w.sum()


def _component_ids(rng: np.random.Generator, n: int, n_comp: int, zipf_s: float | None):
    if zipf_s is None:
        return rng.integers(0, n_comp, size=n)
    w = zipf_weights(n_comp, zipf_s)
    perm = rng.permutation(n_comp)  # which component gets which weight
    return perm[rng.choice(n_comp, size=n, p=w)]


def gaussian_mixture(n: int, d: int, n_comp: int, sigma: float, seed: int,
                     n_query: int = 0, zipf_s: float | None = None):
    """Return (base, query) float32 arrays drawn from one Gaussian mixture."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((n_comp, d))
    comp = _component_ids(rng, n + n_query, n_comp, zipf_s)
    x = centres[comp] + sigma * rng.standard_normal((n + n_query, d))
    x = x.astype(np.float32)
    return x[:n], x[n:]


def sphere_mixture(n: int, d: int, n_comp: int, sigma: float, seed: int,
                   n_query: int = 0, zipf_s: float | None = None):
    """Unit-norm points near random unit-sphere centres (tangent noise)."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((n_comp, d))
    centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    comp = _component_ids(rng, n + n_query, n_comp, zipf_s)
    out = np.empty((n + n_query, d), dtype=np.float32)
    step = 65536
    for s in range(0, n + n_query, step):
        c = centres[comp[s:s + step]]
        noise = rng.standard_normal(c.shape)
        noise -= np.sum(noise * c, axis=1, keepdims=True) * c
        p = c + sigma * noise
        p /= np.linalg.norm(p, axis=1, keepdims=True)
        out[s:s + step] = p
    return out[:n], out[n:]


def kmeans(x: np.ndarray, k: int, iters: int = 20, seed: int = 0):
    """Lloyd's k-means (float64 arithmetic). Returns (centroids f32, ids u32).

    Initial centroids are k distinct points drawn with ``seed``; an empty
    cluster keeps its previous centroid.  The returned ids assign every point
    to its nearest final centroid.
    """
    rng = np.random.default_rng(seed)
    x64 = x.astype(np.float64)
    c = x64[rng.choice(len(x), size=k, replace=False)].copy()

    def assign(cent):
        xx = np.sum(x64 * x64, axis=1)[:, None]
        cc = np.sum(cent * cent, axis=1)[None, :]
        return np.argmin(xx - 2.0 * x64 @ cent.T + cc, axis=1)

    for _ in range(iters):
        a = assign(c)
        sums = np.zeros_like(c)
        np.add.at(sums, a, x64)
        cnt = np.bincount(a, minlength=k)
        nz = cnt > 0
        c[nz] = sums[nz] / cnt[nz, None]
    a = assign(c)
    return c.astype(np.float32), a.astype(np.uint32)


def ground_truth(base: np.ndarray, query: np.ndarray, k: int):
    """Exact top-k by float64 squared L2. Returns (ids u32 [nq,k], dists f64)."""
    b = base.astype(np.float64)
    q = query.astype(np.float64)
    bb = np.sum(b * b, axis=1)
    ids = np.empty((len(q), k), dtype=np.uint32)
    dist = np.empty((len(q), k), dtype=np.float64)
    step = 256
    for s in range(0, len(q), step):
        qq = q[s:s + step]
        d2 = np.sum(qq * qq, axis=1)[:, None] - 2.0 * qq @ b.T + bb[None, :]
        part = np.argpartition(d2, k - 1, axis=1)[:, :k]
        pd = np.take_along_axis(d2, part, axis=1)
        order = np.argsort(pd, axis=1, kind="stable")
        ids[s:s + step] = np.take_along_axis(part, order, axis=1)
        # exact distances of the chosen ids, summed directly
        sel = b[ids[s:s + step]]
        dist[s:s + step] = np.sum((sel - qq[:, None, :]) ** 2, axis=2)
    return ids, dist
