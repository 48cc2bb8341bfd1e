"""Parity with the reference at the headline shape (d = 1536).

Indexes are built by the reference's own create_index (src/create_index.cpp,
compiled by oracle/Makefile) from a seeded unit-sphere mixture - 8-bit
(EX = 7) and 4-bit (EX = 3), 40,000 vectors, K = 128 - and searched on
identical index and rotated-query bytes by the GPU and by the reference's own
IVF::search (inc/index/IVF.hpp:295-324, strict IEEE build
oracle/_ref/liberq_ref.so).  Result ids and distance bits must be equal:
  * erq_search at nprobe 1, 2, 16, 64 and k 10, 100;
  * the batched plan (work-list scan, graph replay);
  * the learned plan, query by query at the depth its model chose.
One query sits exactly on a rotated centroid (y = 0: the unit_q fallback of
normalize_query16, inc/utils/space.hpp:749-778).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CREATE_INDEX = os.path.join(REPO, "oracle", "_ref", "create_index")
N, DIM, K, NQ = 40_000, 1536, 128, 64
NPROBES = (1, 2, 16, 64)


def _reference():
    import oracle

    if not (oracle.reference_available() and os.access(CREATE_INDEX, os.X_OK)):
        pytest.skip("reference build (make -C oracle ref) not present")
    return oracle


@pytest.fixture(scope="module")
def data1536(tmp_path_factory):
    from erq_b200 import datasets, vecs

    work = tmp_path_factory.mktemp("p1536")
    base, query = datasets.sphere_mixture(N, DIM, 256, 0.05, seed=1536, n_query=NQ + 3000)
    cent, ids = datasets.kmeans_torch(torch.from_numpy(base).cuda(), K, iters=10, seed=1537)
    cent = cent.cpu().numpy()
    ids = ids.cpu().numpy().astype(np.int32)
    # keep every member off its centroid: a zero residual makes the reference's
    # fast_quantize run for ~2^31 steps per dimension
    # (inc/index/Quantizer.hpp:142-196)
    rng = np.random.default_rng(1538)
    cent = cent + 1e-3 * rng.standard_normal(cent.shape).astype(np.float32)
    ds = "p1536"
    ddir = work / "data" / ds
    ddir.mkdir(parents=True)
    (work / "bin").mkdir()
    (work / "results" / "indexing_time").mkdir(parents=True)
    vecs.write_vecs(str(ddir / f"{ds}_base.fvecs"), base)
    vecs.write_vecs(str(ddir / f"{ds}_centroid_{K}.fvecs"), cent)
    vecs.write_vecs(str(ddir / f"{ds}_cluster_id_{K}.ivecs"), ids[:, None])
    return work, ds, query


def _index(data1536, bits):
    _reference()
    work, ds, _ = data1536
    path = work / "data" / ds / f"ivf_exhaf{bits}.index"
    if not path.exists():
        subprocess.run([CREATE_INDEX, ds, str(K), str(bits)], cwd=work / "bin", check=True,
                       stdout=subprocess.DEVNULL, timeout=900)
    return str(path)


def _queries(ref, path, query):
    """Rotated by the reference itself; query 3 replaced by a rotated centroid."""
    from erq_b200 import indexfile

    q = ref.rotate(query)
    q[3] = indexfile.read_index(path).centroids[6]
    return q


def _open(path):
    return _reference().Reference(path)  # strict IEEE build


@pytest.mark.parametrize("bits", [8, 4])
def test_search_equals_reference(data1536, bits):
    from erq_b200 import IVF

    path = _index(data1536, bits)
    ref = _open(path)
    assert (ref.D, ref.EX, ref.K) == (DIM, bits - 1, K)
    qrot = _queries(ref, path, data1536[2][:NQ])
    idx = IVF(path)
    for nprobe in NPROBES:
        for k in (10, 100):
            want_ids, want_d = ref.search_dists(qrot, k, nprobe)
            got_ids, got_d = idx.search_batch(qrot, k, nprobe)
            assert (got_ids == want_ids).all(), (bits, nprobe, k)
            assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), (bits, nprobe, k)
    idx.free()
    ref.close()


@pytest.mark.parametrize("bits", [8, 4])
def test_plan_equals_reference(data1536, bits):
    from erq_b200 import IVF, Plan

    path = _index(data1536, bits)
    ref = _open(path)
    qrot = _queries(ref, path, data1536[2][:NQ])
    idx = IVF(path)
    want_ids, want_d = ref.search_dists(qrot, 100, 16)
    plan = Plan(idx, max_batch=NQ, k=100, nprobe=16)
    for tiling in ((1, 16, 4, 4), (2, 8, 8, 32)):
        plan.set_tuning(NQ, *tiling)
        for _ in range(2):  # capture, then replay
            ids, d, _ = plan.search(qrot)
            assert (ids == want_ids).all(), tiling
            assert (d.view(np.uint32) == want_d.view(np.uint32)).all(), tiling
    plan.free()
    idx.free()
    ref.close()


def test_learned_plan_equals_reference_at_chosen_depth(data1536):
    from erq_b200 import IVF, Plan
    from erq_b200.learned import DEFAULT_BINS, ProbeModel, make_labels, probe_features

    path = _index(data1536, 8)
    ref = _open(path)
    query = data1536[2]
    qrot = _queries(ref, path, query[:NQ])
    idx = IVF(path)
    train = idx.rotate(query[NQ:])
    labels = make_labels(idx, train, 100, DEFAULT_BINS)
    model = ProbeModel.train(probe_features(idx, train), labels, DEFAULT_BINS, epochs=20,
                             batch=256, lr=1e-3, seed=3)
    plan = Plan(idx, max_batch=NQ, k=100, nprobe=16, model=model)
    plan.set_learned(0.9, 0.05)
    ids, d, used = plan.search(qrot, with_nprobe=True)
    assert used.min() >= 1 and used.max() <= 16
    for u in np.unique(used):
        sel = np.flatnonzero(used == u)
        want_ids, want_d = ref.search_dists(qrot[sel], 100, int(u))
        assert (ids[sel] == want_ids).all(), int(u)
        assert (d[sel].view(np.uint32) == want_d.view(np.uint32)).all(), int(u)
    plan.free()
    model.free()
    idx.free()
    ref.close()
