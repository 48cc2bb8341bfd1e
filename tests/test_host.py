"""Host-side utilities: fvecs IO, the index file format, metrics, generators."""
import numpy as np
import pytest

from conftest import golden_cases, load_golden
from erq_b200 import datasets, indexfile, metrics, vecs


def test_vecs_roundtrip(tmp_path):
    a = np.random.default_rng(0).standard_normal((7, 13)).astype(np.float32)
    vecs.write_vecs(tmp_path / "a.fvecs", a)
    assert (vecs.read_vecs(tmp_path / "a.fvecs") == a).all()
    b = np.arange(12, dtype=np.uint32).reshape(3, 4)
    vecs.write_vecs(tmp_path / "b.ivecs", b)
    assert (vecs.read_vecs(tmp_path / "b.ivecs", np.uint32) == b).all()


def test_vecs_rejects_ragged(tmp_path):
    raw = np.array([3, 0, 0, 0, 2, 0, 0], np.uint32)
    raw.tofile(tmp_path / "r.fvecs")
    with pytest.raises(ValueError):
        vecs.read_vecs(tmp_path / "r.fvecs")


@pytest.mark.parametrize("name", golden_cases())
def test_index_file_roundtrip(tmp_path, name):
    g = load_golden(name)
    a = indexfile.read_index(g["path"], mmap=False)
    assert a.sizes.sum() == a.N and a.P.shape == (a.D, a.D)
    indexfile.write_index(tmp_path / "x.index", a)
    assert (tmp_path / "x.index").read_bytes() == open(g["path"], "rb").read()


def test_index_file_truncated(tmp_path):
    g = load_golden(golden_cases()[0])
    data = open(g["path"], "rb").read()
    (tmp_path / "t.index").write_bytes(data[:-5])
    with pytest.raises(ValueError):
        indexfile.read_index(tmp_path / "t.index")


def test_recall_counts_like_test_search():
    gt = np.array([[1, 2, 3, 4]], np.uint32)
    res = np.array([[2, 9, 2, 4]], np.uint32)  # repeated id counts twice
    assert metrics.recall_at_k(res, gt, 4) == 3 / 4


def test_distance_ratio_identity():
    rng = np.random.default_rng(1)
    base = rng.standard_normal((50, 8)).astype(np.float32)
    q = rng.standard_normal((3, 8)).astype(np.float32)
    gt, _ = datasets.ground_truth(base, q, 5)
    assert metrics.average_distance_ratio(q, base, gt, gt, 5) == pytest.approx(1.0)


def test_generators_are_seeded_and_shaped():
    a, qa = datasets.sphere_mixture(1000, 32, 16, 0.05, seed=3, n_query=10, zipf_s=1.1)
    b, qb = datasets.sphere_mixture(1000, 32, 16, 0.05, seed=3, n_query=10, zipf_s=1.1)
    assert (a == b).all() and (qa == qb).all() and a.shape == (1000, 32)
    assert np.allclose(np.linalg.norm(a, axis=1), 1.0, atol=1e-5)
    g, _ = datasets.gaussian_mixture(500, 16, 8, 0.3, seed=4)
    assert g.dtype == np.float32 and g.shape == (500, 16)


def test_kmeans_and_ground_truth():
    x, q = datasets.gaussian_mixture(800, 8, 4, 0.1, seed=5, n_query=4)
    c, ids = datasets.kmeans(x, 4, iters=10, seed=0)
    d = ((x[:, None, :].astype(np.float64) - c[None].astype(np.float64)) ** 2).sum(-1)
    assert (ids == d.argmin(1)).all()
    gt, gd = datasets.ground_truth(x, q, 10)
    bf = ((q[:, None, :].astype(np.float64) - x[None].astype(np.float64)) ** 2).sum(-1)
    assert (np.sort(bf, axis=1)[:, :10] == pytest.approx(gd))
