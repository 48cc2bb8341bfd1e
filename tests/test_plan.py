"""Batched search plans (erq_plan_*): the work-list scan, the CUDA graphs and
the autotuner must not change a single result.  Every plan search is checked
bit for bit against erq_search (plain) or erq_search_learned (with a model) on
the same queries: ids and distance bits, for every scan tile shape, several
chunk sizes, several batch sizes, repeated graph replays, raw queries and
device buffers."""
import os

import numpy as np
import pytest

from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SHAPES = [(1, 4), (1, 8), (2, 4), (2, 8), (4, 4), (4, 8)]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("name", golden_cases())
def test_plan_matches_golden(name):
    from erq_b200 import IVF, Plan

    g = load_golden(name)
    idx = IVF(g["path"], device=0)
    k, nprobe = int(g["k"]), int(g["nprobe"])
    ref_ids, ref_d = idx.search_batch(g["qrot"], k, nprobe)
    plan = Plan(idx, max_batch=len(g["qrot"]), k=k, nprobe=nprobe)
    for qb, w in SHAPES:
        plan.set_tuning(len(g["qrot"]), qb, 1, w)
        ids, d, used = plan.search(g["qrot"], with_nprobe=True)
        assert (ids == g["ids"]).all(), (qb, w)
        assert (bits(d) == bits(ref_d)).all(), (qb, w)
        assert (used == min(nprobe, idx.K)).all()
    plan.free()
    idx.free()


@pytest.fixture(scope="module")
def uneven(tmp_path_factory):
    """Clusters = the components of a Zipf-weighted sphere mixture (no
    k-means, which would even them out): from tens of vectors to thousands,
    so work items split into many chunks."""
    from erq_b200 import IVF, build_index, indexfile

    d = tmp_path_factory.mktemp("plan")
    rng = np.random.default_rng(31)
    K, dim, n, nq = 96, 128, 40000, 2000
    w = 1.0 / np.arange(1, K + 1) ** 1.3
    comp = rng.choice(K, size=n + nq, p=w / w.sum())
    centres = rng.standard_normal((K, dim)).astype(np.float32)
    centres /= np.linalg.norm(centres, axis=1, keepdims=True)
    pts = centres[comp] + 0.3 * rng.standard_normal((n + nq, dim)).astype(np.float32)
    pts /= np.linalg.norm(pts, axis=1, keepdims=True)
    base, q, ids = pts[:n], pts[n:], comp[:n]
    present = np.unique(ids)
    remap = np.full(K, -1)
    remap[present] = np.arange(present.size)
    ids = remap[ids]
    cent = np.stack([base[ids == c].mean(0) for c in range(present.size)]).astype(np.float32)
    arr = build_index.build_index_torch(torch.from_numpy(base), torch.from_numpy(cent),
                                        torch.from_numpy(ids.astype(np.int64)), 7, seed=33)
    path = os.path.join(d, "uneven.index")
    indexfile.write_index(path, arr)
    idx = IVF(path)
    sizes = np.bincount(ids, minlength=present.size)
    return idx, q, idx.rotate(q), sizes


def test_uneven_clusters_every_tiling(uneven):
    from erq_b200 import Plan

    idx, q, qr, sizes = uneven
    assert sizes.max() > 20 * sizes.min()  # really uneven
    k, nprobe = 100, 6
    ref_ids, ref_d = idx.search_batch(qr, k, nprobe)
    plan = Plan(idx, max_batch=len(qr), k=k, nprobe=nprobe)
    for qb, w in SHAPES:
        for cb in (1, 3, 16, 64):
            plan.set_tuning(len(qr), qb, cb, w)
            ids, d, _ = plan.search(qr)
            assert (ids == ref_ids).all(), (qb, w, cb)
            assert (bits(d) == bits(ref_d)).all(), (qb, w, cb)
    plan.free()


def test_batch_sizes_and_graph_replays(uneven):
    from erq_b200 import Plan

    idx, q, qr, _ = uneven
    k, nprobe = 50, 4
    plan = Plan(idx, max_batch=1024, k=k, nprobe=nprobe)
    for n in (1, 7, 64, 1024, 7, 1):
        sl = qr[100:100 + n]
        ref_ids, ref_d = idx.search_batch(sl, k, nprobe)
        for _ in range(2):  # second call replays the captured graph
            ids, d, _ = plan.search(sl)
            assert (ids == ref_ids).all(), n
            assert (bits(d) == bits(ref_d)).all(), n
    with pytest.raises(Exception):
        plan.search(qr[:1025])
    plan.free()


def test_both_refinement_forms(uneven):
    """The 4-warp and the wide (32-warp, 128-block window) refinement give the
    same results at batch sizes below and above the SM count, and with k up
    to the largest the pool supports."""
    from erq_b200 import Plan

    idx, q, qr, _ = uneven
    for k, nprobe, n in ((100, 6, 50), (100, 6, 300), (1024, 12, 40)):
        sl = qr[:n]
        ref_ids, ref_d = idx.search_batch(sl, k, nprobe)
        plan = Plan(idx, max_batch=n, k=k, nprobe=nprobe)
        for rw in (4, 32, 0):
            plan.set_tuning(n, 2, 16, 4, rw)
            assert plan.tuning(n)["refine_warps"] == rw
            ids, d, _ = plan.search(sl)
            assert (ids == ref_ids).all(), (k, n, rw)
            assert (bits(d) == bits(ref_d)).all(), (k, n, rw)
        plan.free()


def test_raw_queries_and_device_buffers(uneven):
    from erq_b200 import Plan

    idx, q, qr, _ = uneven
    k, nprobe = 100, 5
    ref_ids, ref_d = idx.search_raw(q[:1500], k, nprobe)
    plan = Plan(idx, max_batch=1500, k=k, nprobe=nprobe, raw=True)
    ids, d, _ = plan.search(q[:1500])
    assert (ids == ref_ids).all()
    assert (bits(d) == bits(ref_d)).all()
    qt = torch.from_numpy(q[:1500]).cuda()
    it = torch.empty((1500, k), dtype=torch.int32, device="cuda")
    dt = torch.empty((1500, k), dtype=torch.float32, device="cuda")
    plan.search_buffers(qt, it, dt)
    torch.cuda.synchronize()
    assert (it.cpu().numpy().view(np.uint32) == ref_ids).all()
    assert (bits(dt.cpu().numpy()) == bits(ref_d)).all()
    plan.free()


def test_autotune_keeps_results(uneven):
    from erq_b200 import Plan

    idx, q, qr, _ = uneven
    k, nprobe = 100, 6
    plan = Plan(idx, max_batch=2000, k=k, nprobe=nprobe)
    t, ms = plan.autotune(qr, reps=1)
    assert t["queries_per_item"] in (1, 2, 4, 8) and t["warps"] in (4, 8) and ms > 0
    assert t["refine_warps"] in (4, 32)
    assert plan.tuning(2000) == t
    ref_ids, ref_d = idx.search_batch(qr, k, nprobe)
    ids, d, _ = plan.search(qr)
    assert (ids == ref_ids).all()
    assert (bits(d) == bits(ref_d)).all()
    plan.free()


def test_learned_plan_equals_learned_search(uneven):
    from erq_b200 import Plan
    from erq_b200.learned import (DEFAULT_BINS, ProbeModel, make_labels, probe_features,
                                  search_learned)

    idx, q, qr, _ = uneven
    k = 100
    labels = make_labels(idx, qr[:1500], k, DEFAULT_BINS)
    model = ProbeModel.train(probe_features(idx, qr[:1500]), labels, DEFAULT_BINS, epochs=5,
                             batch=256, seed=7)
    ev = qr[1500:]
    ids_l, d_l, used_l = search_learned(idx, model, ev, k, nprobe_fallback=6, confidence=0.8)
    plan = Plan(idx, max_batch=len(ev), k=k, nprobe=6, model=model)
    plan.set_learned(0.8)
    for qb, w in ((1, 4), (4, 8)):
        plan.set_tuning(len(ev), qb, 8, w)
        ids, d, used = plan.search(ev, with_nprobe=True)
        assert (used == used_l).all()
        assert (ids == ids_l).all()
        assert (bits(d) == bits(d_l)).all()
    plan.free()
    model.free()


def test_probe_rarely_falls_back(uneven):
    """The coarse probe proves its cut from the estimates with a small margin;
    falling back to all K exact distances must stay rare (a speed property:
    results are exact either way)."""
    from erq_b200 import _lib as L

    idx, q, qr, _ = uneven
    L.probe_fallbacks(0, reset=True)
    idx.search_batch(qr, 100, 6, with_dists=False)
    assert L.probe_fallbacks(0, reset=True) <= 0.02 * len(qr)


def test_host_buffers_pipelined_in_chunks(uneven):
    """A host-buffer batch runs as chunks whose copies overlap the searches
    (two buffer slots, two copy streams); every chunking gives the one-piece
    results, with and without graphs, and repeated calls reuse the slots."""
    from erq_b200 import Plan

    idx, q, qr, _ = uneven
    k, nprobe = 100, 6
    nq = 4099  # odd, so that the chunks differ in size
    rng = np.random.default_rng(41)
    qs = np.ascontiguousarray(qr[rng.integers(0, qr.shape[0], nq)])
    ref_ids, ref_d = idx.search_batch(qs, k, nprobe)
    plan = Plan(idx, max_batch=nq, k=k, nprobe=nprobe)
    qh = torch.from_numpy(qs).pin_memory()
    ids_h = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    d_h = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    u_h = torch.empty(nq, dtype=torch.int32).pin_memory()
    for graphs in (True, False):
        plan.set_graphs(graphs)
        for chunks in (0, 1, 2, 3, 4, 7):
            plan.set_pipeline(chunks)
            for _ in range(2):
                ids_h.fill_(-1)
                d_h.fill_(-1.0)
                plan.search_buffers(qh, ids_h, d_h, u_h)
                assert (ids_h.numpy().view(np.uint32) == ref_ids).all(), (graphs, chunks)
                assert (bits(d_h.numpy()) == bits(ref_d)).all(), (graphs, chunks)
                assert (u_h.numpy() == nprobe).all()
    plan.free()


def test_async_host_buffer_calls(uneven):
    """erq_plan_search_async: consecutive calls alternate buffer slots (the
    copy-in of one overlaps the search of the one before); every call's
    results, read after the stream is synchronised, equal the synchronous
    search's, and a synchronous call after asynchronous ones is ordered."""
    from erq_b200 import Plan

    idx, q, qr, _ = uneven
    k, nprobe, nq = 50, 6, 500
    plan = Plan(idx, max_batch=nq, k=k, nprobe=nprobe)
    st = torch.cuda.current_stream()
    batches = [np.ascontiguousarray(qr[i * nq:(i + 1) * nq]) for i in range(3)]
    want = [idx.search_batch(b, k, nprobe) for b in batches]
    qh = [torch.from_numpy(b).pin_memory() for b in batches]
    outs = [(torch.empty((nq, k), dtype=torch.int32).pin_memory(),
             torch.empty((nq, k), dtype=torch.float32).pin_memory()) for _ in range(6)]
    for c in range(6):
        plan.search_buffers_async(qh[c % 3], outs[c][0], outs[c][1], stream=st)
    torch.cuda.synchronize()
    for c in range(6):
        wi, wd = want[c % 3]
        assert (outs[c][0].numpy().view(np.uint32) == wi).all(), c
        assert (bits(outs[c][1].numpy()) == bits(wd)).all(), c
    plan.search_buffers_async(qh[1], outs[0][0], outs[0][1], stream=st)
    ids, d, _ = plan.search(batches[2])
    torch.cuda.synchronize()
    assert (ids == want[2][0]).all()
    assert (outs[0][0].numpy().view(np.uint32) == want[1][0]).all()
    plan.free()
