"""Learned probing: kernels against a float64 oracle, and what it buys.

* Gradients of the GPU forward/backward kernels match the float64 CPU oracle
  (oracle/mlp_oracle.py) on the same parameters.
* A saved model predicts the same probabilities after loading.
* On a seeded dataset, the learned search returns exactly the plain search's
  results at each query's chosen depth, and reaches the recall of the fixed
  nprobe it replaces with fewer probed clusters on average.
"""
import os

import numpy as np
import pytest

from conftest import ORACLE_DIR  # noqa: F401

torch = pytest.importorskip("torch")


def test_bf16_rounding_matches_torch():
    import mlp_oracle

    x = np.random.default_rng(0).standard_normal(10000).astype(np.float32) * 10
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert (mlp_oracle.to_bf16(x) == ref).all()


@pytest.mark.gpu
def test_gradients_match_fp64_oracle():
    import mlp_oracle
    from erq_b200.learned import ProbeModel

    rng = np.random.default_rng(1)
    f = (rng.standard_normal((1024, 320)) * 3 + 1).astype(np.float32)
    y = rng.integers(0, 8, 1024).astype(np.uint8)
    model = ProbeModel.train(f, y, epochs=2, batch=256, lr=1e-3, seed=3)
    params, mean, std, bins = model.params()
    assert list(bins) == [1, 2, 3, 4, 6, 8, 12, 16]
    fb = (rng.standard_normal((300, 320)) * 3 + 1).astype(np.float32)
    yb = rng.integers(0, 8, 300).astype(np.uint8)
    loss, g = model.grads(fb, yb)
    loss_o, g_o = mlp_oracle.loss_and_grads(params, mean, std, fb, yb)
    assert loss == pytest.approx(loss_o, rel=1e-5)
    # inference runs on tensor cores (split-BF16 activations): probabilities
    # within 1e-4 of the float64 forward pass
    probs = model.predict(fb)
    assert np.abs(probs - mlp_oracle.probabilities(params, mean, std, fb)).max() < 1e-4
    for lo, hi in [(mlp_oracle.W1, mlp_oracle.B1), (mlp_oracle.B1, mlp_oracle.W2),
                   (mlp_oracle.W2, mlp_oracle.B2), (mlp_oracle.B2, mlp_oracle.W3),
                   (mlp_oracle.W3, mlp_oracle.B3), (mlp_oracle.B3, mlp_oracle.N_PARAMS)]:
        a, b = g[lo:hi].astype(np.float64), g_o[lo:hi]
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b) + 1e-9, (lo, hi)
    model.free()


@pytest.mark.gpu
def test_save_load_roundtrip(tmp_path):
    from erq_b200.learned import ProbeModel

    rng = np.random.default_rng(2)
    f = rng.standard_normal((512, 320)).astype(np.float32)
    y = rng.integers(0, 8, 512).astype(np.uint8)
    m = ProbeModel.train(f, y, epochs=3, batch=128, seed=4)
    p1 = m.predict(f[:50])
    m.save(tmp_path / "probe.model")
    m2 = ProbeModel.load(tmp_path / "probe.model")
    p2 = m2.predict(f[:50])
    assert (p1 == p2).all()
    assert np.allclose(p1.sum(1), 1.0, atol=1e-5)


@pytest.fixture(scope="module")
def learned_case(tmp_path_factory):
    from erq_b200 import IVF, build_index, datasets, indexfile

    d = tmp_path_factory.mktemp("learned")
    base, q = datasets.gaussian_mixture(30000, 128, 96, 0.45, seed=21, n_query=9000)
    cent, ids = datasets.kmeans(base, 192, iters=10, seed=22)
    arr = build_index.build_index_torch(torch.from_numpy(base), torch.from_numpy(cent),
                                        torch.from_numpy(ids.astype(np.int64)), 5, seed=23)
    path = os.path.join(d, "learned.index")
    indexfile.write_index(path, arr)
    gt, _ = datasets.ground_truth(base, q[7000:], 100)
    ivf = IVF(path)
    return ivf, ivf.rotate(q[:7000]), ivf.rotate(q[7000:]), gt


@pytest.mark.gpu
def test_learned_search_equals_plain_at_chosen_depth_and_saves_probes(learned_case):
    from erq_b200 import metrics
    from erq_b200.learned import (DEFAULT_BINS, ProbeModel, make_labels, probe_features,
                                  search_learned)

    ivf, rot_train, rot_eval, gt = learned_case
    k = 100
    labels = make_labels(ivf, rot_train, k, DEFAULT_BINS)
    assert len(np.unique(labels)) > 1
    feats = probe_features(ivf, rot_train)
    model = ProbeModel.train(feats, labels, DEFAULT_BINS, epochs=40, batch=512, lr=1e-3, seed=5)
    # fixed nprobe the learned search replaces: smallest depth reaching 95% of
    # the deepest depth's recall
    rec = {}
    for b in DEFAULT_BINS:
        ids_b, _ = ivf.search_batch(rot_eval, k, b, with_dists=False)
        rec[b] = metrics.recall_at_k(ids_b, gt, k)
    target = 0.95 * rec[DEFAULT_BINS[-1]]
    fixed = next(b for b in DEFAULT_BINS if rec[b] >= target)
    ids, d, used = search_learned(ivf, model, rot_eval, k, nprobe_fallback=fixed,
                                  confidence=0.9)
    # exactness: each query's result is the plain search's at its depth
    for u in np.unique(used):
        sel = np.flatnonzero(used == u)
        ids_u, d_u = ivf.search_batch(rot_eval[sel], k, int(u))
        assert (ids[sel] == ids_u).all()
        assert (d[sel].view(np.uint32) == d_u.view(np.uint32)).all()
    r_learned = metrics.recall_at_k(ids, gt, k)
    print(f"fixed nprobe {fixed}: recall {rec[fixed]:.4f}; learned: mean nprobe "
          f"{used.mean():.2f}, recall {r_learned:.4f}")
    assert r_learned >= rec[fixed] - 0.01
    assert used.mean() < fixed


@pytest.mark.gpu
def test_distance_features_follow_exact_centroid_distances(learned_case):
    """The 64 distance features come from the tensor-core estimates; they must
    agree with the same features computed from the exact distances."""
    from erq_b200.learned import probe_features

    ivf, rot_train, _, _ = learned_case
    q = rot_train[:200]
    f = probe_features(ivf, q)
    exact = np.sort(ivf.debug_centroid_dists(q).astype(np.float64), axis=1)[:, :64]
    qn = (q.astype(np.float64) ** 2).sum(1)
    ref = np.concatenate([np.log(exact[:, :1] / qn[:, None] + 1e-12),
                          exact[:, 1:] / exact[:, :1] - 1.0], axis=1)
    assert np.abs(f[:, 256:] - ref).max() < 1e-3
    sketch = np.zeros((q.shape[0], 256))
    d = min(256, q.shape[1])  # dims beyond D read as 0
    sketch[:, :d] = q[:, :d] * (16.0 / np.sqrt(qn))[:, None]
    assert np.abs(f[:, :256] - sketch).max() < 1e-4
