"""Result-quality metrics of the reference's test_search (src/test_search.cpp:113-124)."""
from __future__ import annotations

import numpy as np


def recall_at_k(results: np.ndarray, gt: np.ndarray, k: int) -> float:
    """Fraction of returned ids found in the first k ground-truth ids, counted
    per returned slot as test_search does (a repeated id counts each time)."""
    res = np.asarray(results)[:, :k].astype(np.int64)
    g = np.asarray(gt)[:, :k].astype(np.int64)
    hits = sum(int(np.isin(r, t).sum()) for r, t in zip(res, g))
    return hits / float(res.shape[0] * k)


def average_distance_ratio(query: np.ndarray, base: np.ndarray, results: np.ndarray,
                           gt: np.ndarray, k: int) -> float:
    """Mean over queries of get_ratio (inc/utils/tools.hpp:16-51) divided by k:
    sqrt(ann_dist / gt_dist) rank by rank (both sorted), skipping gt
    distances <= 1e-5; distances are squared L2 in float64."""
    total = 0.0
    for qi in range(query.shape[0]):
        q = query[qi].astype(np.float64)
        g = np.sort(np.sum((base[gt[qi, :k]].astype(np.float64) - q) ** 2, axis=1))
        a = np.sort(np.sum((base[results[qi, :k]].astype(np.float64) - q) ** 2, axis=1))
        valid = g > 1e-5
        if not np.any(valid):
            total += 1.0
            continue
        total += float(np.mean(np.sqrt(a[valid] / g[valid])))
    return total / query.shape[0]
