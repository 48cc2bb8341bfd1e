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


# ---------------------------------------------------------------- GPU versions
# torch is used here as data-preparation plumbing for the large workloads
# (generation, clustering, ground truth); the search itself never uses it.

def sphere_mixture_torch(n: int, d: int, n_comp: int, sigma: float, seed: int,
                         n_query: int = 0, zipf_s: float | None = None, device="cuda"):
    """GPU twin of ``sphere_mixture`` (same distribution, different stream)."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)
    centres = torch.randn(n_comp, d, generator=g, device=device)
    centres /= centres.norm(dim=1, keepdim=True)
    if zipf_s is None:
        comp = torch.randint(0, n_comp, (n + n_query,), generator=g, device=device)
    else:
        w = torch.tensor(zipf_weights(n_comp, zipf_s), device=device)
        perm = torch.randperm(n_comp, generator=g, device=device)
        comp = perm[torch.multinomial(w, n + n_query, replacement=True, generator=g)]
    out = torch.empty(n + n_query, d, device=device)
    step = 1 << 17
    for s in range(0, n + n_query, step):
        c = centres[comp[s:s + step]]
        noise = torch.randn(c.shape, generator=g, device=device)
        noise -= (noise * c).sum(1, keepdim=True) * c
        p = c + sigma * noise
        out[s:s + step] = p / p.norm(dim=1, keepdim=True)
    return out[:n], out[n:]


def gaussian_mixture_torch(n: int, d: int, n_comp: int, sigma: float, seed: int,
                           n_query: int = 0, zipf_s: float | None = None, device="cuda"):
    """GPU twin of ``gaussian_mixture``; Zipf(zipf_s) component weights when
    given (the weights assigned to components in a seeded random order)."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)
    centres = torch.randn(n_comp, d, generator=g, device=device)
    if zipf_s is None:
        comp = torch.randint(0, n_comp, (n + n_query,), generator=g, device=device)
    else:
        w = torch.from_numpy(zipf_weights(n_comp, zipf_s)).to(device)
        perm = torch.randperm(n_comp, generator=g, device=device)
        comp = perm[torch.multinomial(w, n + n_query, replacement=True, generator=g)]
    x = torch.empty(n + n_query, d, device=device)
    step = 1 << 20
    for s in range(0, n + n_query, step):
        c = comp[s:s + step]
        x[s:s + step] = centres[c] + sigma * torch.randn(c.numel(), d, generator=g, device=device)
    return x[:n], x[n:]


def ground_truth_shortlist(base, query, k: int, shortlist: int = 1024, qstep: int = 1024,
                           bstep: int = 1 << 20):
    """Top-k by squared L2 for large bases: a TF32 distance pass keeps the
    ``shortlist`` nearest per query, which are then ranked exactly in float64.
    Returns (ids int64 [nq, k], dists float64 [nq, k])."""
    import torch

    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    try:
        nq = query.shape[0]
        cand_d = torch.full((nq, shortlist), float("inf"), device=base.device)
        cand_i = torch.zeros((nq, shortlist), dtype=torch.long, device=base.device)
        for b0 in range(0, base.shape[0], bstep):
            b = base[b0:b0 + bstep]
            bb = (b * b).sum(1)
            for q0 in range(0, nq, qstep):
                q = query[q0:q0 + qstep]
                d = bb[None, :] - 2.0 * (q @ b.T)
                kk = min(shortlist, d.shape[1])
                vd, vi = d.topk(kk, dim=1, largest=False)
                cd = torch.cat([cand_d[q0:q0 + qstep], vd], 1)
                ci = torch.cat([cand_i[q0:q0 + qstep], vi + b0], 1)
                o = cd.topk(shortlist, dim=1, largest=False).indices
                cand_d[q0:q0 + qstep] = cd.gather(1, o)
                cand_i[q0:q0 + qstep] = ci.gather(1, o)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    best_i = torch.empty((nq, k), dtype=torch.long, device=base.device)
    best_d = torch.empty((nq, k), dtype=torch.float64, device=base.device)
    rstep = 128
    for q0 in range(0, nq, rstep):
        q = query[q0:q0 + rstep].double()
        ci = cand_i[q0:q0 + rstep]
        ex = ((base[ci].double() - q[:, None, :]) ** 2).sum(2)
        o = torch.argsort(ex, dim=1, stable=True)[:, :k]
        best_i[q0:q0 + rstep] = ci.gather(1, o)
        best_d[q0:q0 + rstep] = ex.gather(1, o)
    return best_i, best_d


def kmeans_torch(x, k: int, iters: int = 20, seed: int = 0):
    """Lloyd's k-means on the GPU (TF32 distance products, float32 updates).
    Returns (centroids [k, d] float32, ids [n] int64) with ids the nearest
    final centroid.  Deterministic algorithms are on while it runs (the
    centroid sums otherwise depend on the order of float atomics), so the same
    seed gives the same clusters on every run."""
    import torch

    g = torch.Generator(device=x.device).manual_seed(seed)
    c = x[torch.randperm(x.shape[0], generator=g, device=x.device)[:k]].clone()
    prev = torch.backends.cuda.matmul.allow_tf32
    prev_det = torch.are_deterministic_algorithms_enabled()
    prev_warn = torch.is_deterministic_algorithms_warn_only_enabled()
    torch.backends.cuda.matmul.allow_tf32 = True
    torch.use_deterministic_algorithms(True, warn_only=True)
    try:
        def assign(cent):
            cc = (cent * cent).sum(1)
            ids = torch.empty(x.shape[0], dtype=torch.long, device=x.device)
            step = 1 << 16
            for s in range(0, x.shape[0], step):
                xs = x[s:s + step]
                ids[s:s + step] = (cc[None, :] - 2.0 * xs @ cent.T).argmin(1)
            return ids

        rng = np.random.default_rng(seed)
        for _ in range(iters):
            a = assign(c)
            sums = torch.zeros_like(c).index_add_(0, a, x)
            cnt = torch.bincount(a, minlength=k)
            nz = cnt > 0
            c[nz] = sums[nz] / cnt[nz, None].to(x.dtype)
            _split_empty_clusters(c, cnt.cpu().numpy(), rng)
        a = assign(c)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
        torch.use_deterministic_algorithms(prev_det, warn_only=prev_warn)
    return c, a


def _split_empty_clusters(c, counts, rng, eps: float = 1.0 / 1024):
    """Re-seed every empty cluster by splitting a populated one, chosen with
    probability proportional to its size: the two centroids become the old
    one scaled by (1 +- eps) alternately per dimension and the members are
    shared (the empty-cluster rule of faiss's k-means, which the reference's
    clustering step uses, python/ivf.py)."""
    import torch

    counts = counts.astype(np.float64).copy()
    empty = np.flatnonzero(counts == 0)
    if empty.size == 0:
        return
    n, k = counts.sum(), counts.size
    sign = torch.ones(c.shape[1], device=c.device, dtype=c.dtype)
    sign[1::2] = -1.0
    for ci in empty:
        p = np.maximum(counts - 1.0, 0.0)
        p /= p.sum() if p.sum() > 0 else 1.0
        cj = int(rng.choice(k, p=p)) if p.sum() > 0 else int(np.argmax(counts))
        c[ci] = c[cj] * (1 + eps * sign)
        c[cj] = c[cj] * (1 - eps * sign)
        counts[ci] = counts[cj] / 2
        counts[cj] -= counts[ci]
    del n


def ground_truth_torch(base, query, k: int, qstep: int = 2048, bstep: int = 1 << 18):
    """Exact top-k by float64 squared L2 on the GPU.  Returns (ids int64
    [nq, k], dists float64 [nq, k])."""
    import torch

    nq = query.shape[0]
    best_d = torch.full((nq, k), float("inf"), dtype=torch.float64, device=base.device)
    best_i = torch.zeros((nq, k), dtype=torch.long, device=base.device)
    for b0 in range(0, base.shape[0], bstep):
        b = base[b0:b0 + bstep].double()
        bb = (b * b).sum(1)
        for q0 in range(0, nq, qstep):
            q = query[q0:q0 + qstep].double()
            d = (q * q).sum(1, keepdim=True) - 2.0 * q @ b.T + bb[None, :]
            kk = min(k, d.shape[1])
            vd, vi = d.topk(kk, dim=1, largest=False)
            cat_d = torch.cat([best_d[q0:q0 + qstep], vd], 1)
            cat_i = torch.cat([best_i[q0:q0 + qstep], vi + b0], 1)
            o = torch.argsort(cat_d, dim=1, stable=True)[:, :k]
            best_d[q0:q0 + qstep] = cat_d.gather(1, o)
            best_i[q0:q0 + qstep] = cat_i.gather(1, o)
    # exact distances of the selected ids, summed directly in float64
    for q0 in range(0, nq, qstep):
        q = query[q0:q0 + qstep].double()
        sel = base[best_i[q0:q0 + qstep]].double()
        best_d[q0:q0 + qstep] = ((sel - q[:, None, :]) ** 2).sum(2)
    return best_i, best_d
