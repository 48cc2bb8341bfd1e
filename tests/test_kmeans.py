"""IVF clustering (erq_kmeans*, kmeans.cuh) against the CPU restatement in
oracle/kmeans_oracle.py.

One Lloyd step from the same centroids: every point goes to its nearest
centroid except where the two nearest are closer than the estimate's error
bound (distances on the tensor cores are split-BF16 products, about FP32
accuracy: 1e-5 of ||x||^2 + ||c||^2 is allowed); the new centroids equal the
float64 means of the GPU's assignment within 1e-6 (relative to the largest
coordinate) and the empty clusters are split as the restatement splits them.
The full run is deterministic and its clusters are the nearest-centroid
partition of its own centroids."""
import numpy as np
import pytest

from conftest import ORACLE_DIR  # noqa: F401  (oracle/ on sys.path)


def test_splitmix64_known_answer():
    from kmeans_oracle import SplitMix64

    r = SplitMix64(0)
    assert r.next() == 0xE220A8397B1DCDAF
    assert r.next() == 0x6E789E6AA1B965F4


def _data(n, dim, comps, seed):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((comps, dim))
    x = c[rng.integers(0, comps, n)] + 0.3 * rng.standard_normal((n, dim))
    return x.astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("n,dim,k", [(20000, 64, 256), (6000, 100, 97), (30000, 1536, 64)])
def test_step_equals_restatement(n, dim, k):
    from kmeans_oracle import exact_dists, update

    from erq_b200.clustering import kmeans_step

    x = _data(n, dim, 32, n + dim)
    rng = np.random.default_rng(k)
    c0 = x[rng.choice(n, k, replace=False)].copy()
    c0[: k // 8] += 100.0  # far centroids: some clusters come out empty
    c1, assign, counts = kmeans_step(x, c0, seed=77)
    d = exact_dists(x, c0)
    best = d.argmin(1)
    srt = np.sort(d, 1)
    bound = 1e-5 * ((x.astype(np.float64) ** 2).sum(1) + (c0.astype(np.float64) ** 2).sum(1).max())
    near_tie = (srt[:, 1] - srt[:, 0]) <= bound
    ok = (assign == best) | near_tie
    assert ok.all(), int((~ok).sum())
    assert (assign[~near_tie] == best[~near_tie]).all()
    # the chosen centroid is within the bound of the nearest
    assert (d[np.arange(n), assign] - srt[:, 0] <= bound).all()
    assert (counts == np.bincount(assign, minlength=k)).all()
    assert (counts == 0).any()  # the split path ran
    want, _ = update(x, assign.astype(np.int64), c0, seed=77)
    tol = 1e-6 * np.abs(x).max()
    assert np.abs(c1 - want).max() <= tol, float(np.abs(c1 - want).max())


@pytest.mark.gpu
def test_full_run_is_deterministic_and_consistent():
    from kmeans_oracle import exact_dists, init_rows

    from erq_b200.clustering import kmeans

    x = _data(40000, 96, 64, 5)
    c1, a1 = kmeans(x, 200, iters=8, seed=11)
    c2, a2 = kmeans(x, 200, iters=8, seed=11)
    assert (c1.view(np.uint32) == c2.view(np.uint32)).all()
    assert (a1 == a2).all()
    d = exact_dists(x, c1)
    srt = np.sort(d, 1)
    bound = 1e-5 * ((x.astype(np.float64) ** 2).sum(1) + (c1.astype(np.float64) ** 2).sum(1).max())
    assert (d[np.arange(x.shape[0]), a1] - srt[:, 0] <= bound).all()
    assert np.bincount(a1, minlength=200).min() > 0
    # zero iterations: the centroids are the seeded initial rows
    c0, _ = kmeans(x, 200, iters=0, seed=11)
    assert (c0 == x[init_rows(x.shape[0], 200, 11)]).all()
