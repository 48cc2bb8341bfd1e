"""The reference's second index format: without HIGH_ACC_FAST_SCAN its
builder writes four factors per vector in each FastScan block and its search
runs Searcher (inc/index/Searcher.hpp) - a 14-bit unsigned query quantisation
over [vl, vr], a different lower bound, a lane-by-lane candidate test
(lower <= the running k-th distance) and a float distance formula on the
residual.  The indexes here are built by the reference's own IVF::construct
compiled without that define (oracle/ref_lowacc.cpp), for every EX width, and
the GPU's ids and distance bits must equal the reference Searcher's."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _lowacc():
    import oracle

    if not oracle.LowAccReference.available():
        pytest.skip("reference build (make -C oracle ref) not present")
    return oracle.LowAccReference


def _build(tmp_path, dim, bits, n=3000, K=24, nq=16, seed=0):
    from erq_b200 import datasets

    L = _lowacc()
    base, query = datasets.gaussian_mixture(n, dim, 16, 0.3, seed=seed + bits, n_query=nq)
    cent, ids = datasets.kmeans(base, K, iters=5, seed=seed + 1)
    # members off their centroids (fast_quantize, inc/index/Quantizer.hpp:142-196)
    cent = cent + 0.01 * np.random.default_rng(seed + 2).standard_normal(cent.shape).astype(np.float32)
    path = str(tmp_path / f"low_d{dim}_b{bits}.index")
    L.build(base, cent, ids.astype(np.uint32), bits, path)
    ref = L(path)
    return path, ref, ref.rotate(query)


@pytest.mark.parametrize("bits", [3, 4, 5, 7, 8, 9])
def test_lowacc_search_equals_reference(tmp_path, bits):
    from erq_b200 import IVF

    path, ref, qrot = _build(tmp_path, 100, bits)
    idx = IVF(path)
    assert idx.block_factors == 4 and idx.EX_BITS == bits - 1
    for k, nprobe in ((10, 1), (50, 6), (100, 24)):
        want_ids, want_d = ref.search_dists(qrot, k, nprobe)
        got_ids, got_d = idx.search_batch(qrot, k, nprobe)
        assert (got_ids == want_ids).all(), (bits, k, nprobe)
        assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), (bits, k, nprobe)
    idx.free()
    ref.close()


def test_lowacc_headline_shape(tmp_path):
    """d = 1536, 8-bit (EX = 7)."""
    from erq_b200 import IVF, load_library

    path, ref, qrot = _build(tmp_path, 1536, 8, n=8000, K=32, nq=12, seed=7)
    idx = IVF(path)
    for k, nprobe in ((100, 2), (100, 16)):
        want_ids, want_d = ref.search_dists(qrot, k, nprobe)
        got_ids, got_d = idx.search_batch(qrot, k, nprobe)
        assert (got_ids == want_ids).all(), nprobe
        assert (got_d.view(np.uint32) == want_d.view(np.uint32)).all(), nprobe
    # the allocation-free entry point runs the same format
    lib = load_library()
    q = torch.from_numpy(qrot).cuda()
    ids = torch.empty((q.shape[0], 100), dtype=torch.int32, device="cuda")
    d = torch.empty((q.shape[0], 100), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    assert lib.erq_search_noalloc(idx._h, C.c_void_p(q.data_ptr()), q.shape[0], 100, 16,
                                  C.c_void_p(ids.data_ptr()), C.c_void_p(d.data_ptr()),
                                  C.c_void_p(st.cuda_stream)) == 0, lib.erq_last_error()
    torch.cuda.synchronize()
    assert (ids.cpu().numpy().view(np.uint32) == got_ids).all()
    assert (d.cpu().numpy().view(np.uint32) == got_d.view(np.uint32)).all()
    idx.free()
    ref.close()


def test_plans_refuse_the_lowacc_format(tmp_path):
    from erq_b200 import IVF, Plan
    from erq_b200._lib import ErqError

    path, ref, _ = _build(tmp_path, 64, 4)
    idx = IVF(path)
    with pytest.raises(ErqError, match="HIGH_ACC_FAST_SCAN"):
        Plan(idx, max_batch=8, k=10, nprobe=2)
    idx.free()
    ref.close()
    assert os.path.exists(path)
