"""Indexes with many clusters.

The reference probes with FlatInitializer for every K < 20000
(inc/index/IVF.hpp:157-161, inc/index/Initializer.hpp:55-68) and with an HNSW
graph over the centroids from K = 20000 on.  Here:
  * K = 19,999 (the largest Flat index), built by the reference's own
    create_index: results equal the reference's IVF::search (strict build) at
    small and at very large nprobe (17,000: the selection and the exact
    top-nprobe sort leave shared memory for global memory);
  * K = 24,000: the loader ignores the HNSW side file and probes every K
    exactly, so results equal the C restatement of the Flat search;
  * the allocation-free entry point agrees with erq_search at both K.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CREATE_INDEX = os.path.join(REPO, "oracle", "_ref", "create_index")
DIM, N, NQ = 64, 60_000, 24


def _data(K, seed):
    rng = np.random.default_rng(seed)
    base = rng.standard_normal((N, DIM)).astype(np.float32)
    query = rng.standard_normal((NQ, DIM)).astype(np.float32)
    # clusters: every K non-empty, the rest at random; centroids = member
    # means moved off their members (a zero residual stalls the reference's
    # fast_quantize, inc/index/Quantizer.hpp:142-196)
    ids = np.concatenate([np.arange(K), rng.integers(0, K, N - K)])
    rng.shuffle(ids)
    cnt = np.bincount(ids, minlength=K).astype(np.float64)
    cent = np.zeros((K, DIM))
    np.add.at(cent, ids, base.astype(np.float64))
    cent = (cent / cnt[:, None]).astype(np.float32)
    cent += 0.01 * rng.standard_normal(cent.shape).astype(np.float32)
    return base, query, cent, ids.astype(np.int32)


def _noalloc(idx, qrot, k, nprobe):
    from erq_b200 import load_library

    lib = load_library()
    q = torch.from_numpy(np.ascontiguousarray(qrot)).cuda()
    ids = torch.empty((q.shape[0], k), dtype=torch.int32, device="cuda")
    d = torch.empty((q.shape[0], k), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    rc = lib.erq_search_noalloc(idx._h, C.c_void_p(q.data_ptr()), q.shape[0], k, nprobe,
                                C.c_void_p(ids.data_ptr()), C.c_void_p(d.data_ptr()),
                                C.c_void_p(st.cuda_stream))
    assert rc == 0, lib.erq_last_error()
    torch.cuda.synchronize()
    return ids.cpu().numpy().view(np.uint32), d.cpu().numpy()


def test_k19999_equals_reference(tmp_path):
    import oracle

    from erq_b200 import IVF, vecs

    if not (oracle.reference_available() and os.access(CREATE_INDEX, os.X_OK)):
        pytest.skip("reference build (make -C oracle ref) not present")
    K = 19_999
    base, query, cent, ids = _data(K, 19999)
    ds = "k19999"
    ddir = tmp_path / "data" / ds
    ddir.mkdir(parents=True)
    (tmp_path / "bin").mkdir()
    (tmp_path / "results" / "indexing_time").mkdir(parents=True)
    vecs.write_vecs(str(ddir / f"{ds}_base.fvecs"), base)
    vecs.write_vecs(str(ddir / f"{ds}_centroid_{K}.fvecs"), cent)
    vecs.write_vecs(str(ddir / f"{ds}_cluster_id_{K}.ivecs"), ids[:, None])
    subprocess.run([CREATE_INDEX, ds, str(K), "4"], cwd=tmp_path / "bin", check=True,
                   stdout=subprocess.DEVNULL, timeout=900)
    path = str(ddir / "ivf_exhaf4.index")
    ref = oracle.Reference(path)
    assert ref.K == K
    qrot = ref.rotate(query)
    idx = IVF(path)
    for k, nprobe in ((10, 1), (100, 64), (100, 17_000)):
        want_ids, want_d = ref.search_dists(qrot, k, nprobe)
        got_ids, got_d = idx.search_batch(qrot, k, nprobe)
        assert (got_ids == want_ids).all(), nprobe
        assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), nprobe
        na_ids, na_d = _noalloc(idx, qrot[:4], k, nprobe)
        assert (na_ids == got_ids[:4]).all(), nprobe
        assert (na_d.view(np.uint32) == got_d[:4].view(np.uint32)).all(), nprobe
    idx.free()
    ref.close()


def test_k24000_probes_exactly(tmp_path, oracle_mod):
    from erq_b200 import IVF, build_index, indexfile

    K = 24_000
    base, query, cent, ids = _data(K, 24000)
    arr = build_index.build_index_torch(torch.from_numpy(base).cuda(), torch.from_numpy(cent).cuda(),
                                        torch.from_numpy(ids.astype(np.int64)).cuda(), 5, seed=5)
    path = str(tmp_path / "k24000.index")
    indexfile.write_index(path, arr)
    idx = IVF(path)
    assert idx.K == K
    qrot = idx.rotate(query)
    o = oracle_mod.Oracle(path)
    for k, nprobe in ((10, 1), (100, 200), (50, 20_000)):
        want_ids, want_d = o.search(qrot, k, nprobe, nthreads=8)
        got_ids, got_d = idx.search_batch(qrot, k, nprobe)
        assert (got_ids == want_ids).all(), nprobe
        assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), nprobe
        na_ids, na_d = _noalloc(idx, qrot[:4], k, nprobe)
        assert (na_ids == got_ids[:4]).all(), nprobe
        assert (na_d.view(np.uint32) == got_d[:4].view(np.uint32)).all(), nprobe
    o.close()
    idx.free()
