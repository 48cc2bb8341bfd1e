"""GPU search through the C ABI against the reference's outputs.

Integer and index work must be bit-exact; floating-point stages that the
reference evaluates in a fixed order (centroid distances, unit_q, delta,
sumq, the per-lane estimates, refined distances) must also match bit for bit
because the kernels follow the same order.  The only tolerance is the query
rotation (a GEMM whose summation order differs from the reference's): it is
checked against a float64 product within 1e-5 relative.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module", params=golden_cases())
def case(request):
    from erq_b200 import IVF

    g = load_golden(request.param)
    idx = IVF(g["path"], device=0)
    yield g, idx
    idx.free()


def test_load_info(case):
    g, idx = case
    from erq_b200 import indexfile

    a = indexfile.read_index(g["path"])
    assert (idx.N, idx.DIM, idx.D, idx.K, idx.EX_BITS) == (a.N, a.DIM, a.D, a.K, a.EX)
    assert idx.padded_dim() == a.D and idx.k() == a.K


def test_centroid_distances_bit_exact(case):
    g, idx = case
    d = idx.debug_centroid_dists(g["qrot"])
    assert (bits(d) == bits(g["centroid_dists"])).all()


def test_probe_lists(case):
    g, idx = case
    cids, sq = idx.debug_probe(g["qrot"], int(g["nprobe"]))
    assert (cids == g["probe_cids"]).all()
    assert (bits(sq) == bits(g["probe_sqy"])).all()


def test_scan_sums_bit_exact(case, oracle_mod):
    g, idx = case
    nprobe = int(g["nprobe"])
    r = idx.debug_scan(g["qrot"], nprobe)
    assert (r["cids"] == g["probe_cids"]).all()
    assert (bits(r["delta"]) == bits(g["delta"])).all()
    assert (bits(r["sumq"]) == bits(g["sumq"])).all()
    o = oracle_mod.Oracle(g["path"])
    sizes = o.cluster_sizes()
    k = 0
    for qi in range(g["qrot"].shape[0]):
        for p in range(nprobe):
            cid = int(r["cids"][qi, p])
            n = int(sizes[cid])
            nb = (n + 31) // 32
            off = int(r["offsets"][qi, p])
            S = r["S"][off:off + 32 * nb]
            S_o, _, _ = o.scan_cluster(g["qrot"][qi], cid, g["probe_sqy"][qi, p], np.float32(np.inf))
            valid = np.arange(32 * nb) < n
            assert (S[valid] == S_o[valid]).all()
            lo, hi = g["ipq_off"][k], g["ipq_off"][k + 1]
            ipq = (S.astype(np.float32) * g["delta"][qi, p]).astype(np.float32)
            assert (bits(ipq)[valid] == bits(g["ipq"][lo:hi])[valid]).all()
            k += 1
    o.close()


def test_search_matches_reference(case):
    g, idx = case
    ids, d = idx.search_batch(g["qrot"], int(g["k"]), int(g["nprobe"]))
    assert (ids == g["ids"]).all()
    assert (bits(d) == bits(g["dists"])).all()


def test_single_query_reference_signature(case):
    g, idx = case
    k = int(g["k"])
    res = np.zeros(k, np.uint32)
    idx.search(g["qrot"][0], None, k, int(g["nprobe"]), res)
    assert (res == g["ids"][0]).all()


def test_search_device_tensors(case):
    torch = pytest.importorskip("torch")
    g, idx = case
    q = torch.from_numpy(g["qrot"]).cuda()
    ids, d = idx.search_batch(q, int(g["k"]), int(g["nprobe"]),
                              stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    assert (ids.cpu().numpy().view(np.uint32) == g["ids"]).all()
    assert (bits(d.cpu().numpy()) == bits(g["dists"])).all()


def test_every_nprobe_and_k_match_oracle(case, oracle_mod):
    """Sweep nprobe 1..K (capped) and several k against the C oracle."""
    g, idx = case
    o = oracle_mod.Oracle(g["path"])
    q = g["qrot"][:4]
    for nprobe in sorted({1, 2, int(g["nprobe"]), max(1, idx.K // 2), idx.K}):
        for k in (1, 7, 33, 100):
            ids, d = idx.search_batch(q, k, nprobe)
            io, do = o.search(q, k, nprobe)
            assert (ids == io).all(), (nprobe, k)
            assert (bits(d) == bits(do)).all(), (nprobe, k)
    o.close()


def test_refine_candidate_count(case, oracle_mod):
    """The refinement's candidate counter equals the number of EX-bit
    distances the reference computes (the oracle's trace length)."""
    from erq_b200 import _lib as L

    g, idx = case
    o = oracle_mod.Oracle(g["path"])
    q = g["qrot"]
    k, nprobe = int(g["k"]), int(g["nprobe"])
    L.refine_stats(0, enable=True)
    idx.search_batch(q, k, nprobe)
    st = L.refine_stats(0, enable=False)
    want = sum(len(o.trace(q[i], k, nprobe)[0]) for i in range(q.shape[0]))
    assert st["candidates"] == want
    assert want <= st["refined"] <= 32 * st["blocks"] and st["windows"] > 0
    idx.search_batch(q, k, nprobe)  # counting off: nothing added
    assert L.refine_stats(0, enable=False) == dict.fromkeys(st, 0)
    o.close()


def test_rotation_accuracy(case):
    g, idx = case
    from erq_b200 import indexfile

    a = indexfile.read_index(g["path"])
    rng = np.random.default_rng(0)
    raw = rng.standard_normal((37, idx.DIM)).astype(np.float32)
    rot = idx.rotate(raw)
    pad = np.zeros((37, idx.D), np.float64)
    pad[:, :idx.DIM] = raw
    ref = pad @ a.P.astype(np.float64)
    scale = np.abs(pad) @ np.abs(a.P.astype(np.float64))
    assert np.all(np.abs(rot - ref) <= 1e-5 * scale + 1e-30)
    # rotate-then-search equals search on the same rotated bytes
    ids_raw, d_raw = idx.search_raw(raw, 10, 3)
    ids, d = idx.search_batch(rot, 10, 3)
    assert (ids_raw == ids).all() and (bits(d_raw) == bits(d)).all()


def test_many_queries_against_oracle(oracle_mod):
    """A few thousand perturbed-centroid queries on the largest golden index."""
    from erq_b200 import IVF

    name = max(golden_cases(), key=lambda n: load_golden(n)["qrot"].shape[1])
    g = load_golden(name)
    idx = IVF(g["path"])
    o = oracle_mod.Oracle(g["path"])
    rng = np.random.default_rng(7)
    cent = o.centroids()
    q = (cent[rng.integers(0, o.K, 3000)] +
         0.2 * rng.standard_normal((3000, o.D))).astype(np.float32)
    ids, d = idx.search_batch(q, 100, 8)
    io, do = o.search(q, 100, 8, nthreads=8)
    assert (ids == io).all()
    assert (bits(d) == bits(do)).all()
    idx.free()
    o.close()


def test_errors_are_reported(tmp_path):
    from erq_b200 import IVF, ErqError

    g = load_golden(golden_cases()[0])
    idx = IVF(g["path"])
    with pytest.raises(ErqError, match="INVALID_ARGUMENT"):
        idx.search_batch(g["qrot"], 10, idx.K + 1)
    with pytest.raises(ErqError, match="INVALID_ARGUMENT"):
        idx.search_batch(g["qrot"], 2000, 2)
    with pytest.raises(ErqError, match="ERR_IO"):
        IVF(str(tmp_path / "missing.index"))
    data = open(g["path"], "rb").read()
    (tmp_path / "trunc.index").write_bytes(data[: len(data) // 2])
    with pytest.raises(ErqError, match="FORMAT"):
        IVF(str(tmp_path / "trunc.index"))
    # K >= 20000 as the reference writes it: the centroids only in the hnswlib
    # side file (inc/index/Initializer.hpp:117-121), so the main file lacks
    # the K x D centroid block - refused with a clear status
    K, D, N, EX = 20000, 64, 20000, 3
    body = (np.array([N, D, K, EX], np.uint64).tobytes() + np.ones(K, np.uint64).tobytes()
            + bytes(D * D * 4 + K * (4 * D + 128) + N * (D * EX // 8 + 8)))
    (tmp_path / "hnsw.index").write_bytes(body)
    with pytest.raises(ErqError, match="UNSUPPORTED.*side file"):
        IVF(str(tmp_path / "hnsw.index"))
    # the handle still works after the failed calls
    ids, _ = idx.search_batch(g["qrot"], int(g["k"]), int(g["nprobe"]))
    assert (ids == g["ids"]).all()
    idx.free()


def test_probe_lists_many_queries(oracle_mod):
    """Tensor-core estimates + exact recompute give the reference's probe
    lists for thousands of queries, including queries at a centroid and
    queries equidistant from several centroids."""
    from erq_b200 import IVF

    for name in golden_cases():
        g = load_golden(name)
        idx = IVF(g["path"])
        o = oracle_mod.Oracle(g["path"])
        cent = o.centroids()
        rng = np.random.default_rng(3)
        n = 1500
        q = (cent[rng.integers(0, o.K, n)] + rng.choice([0.0, 0.05, 0.5], size=(n, 1)) *
             rng.standard_normal((n, o.D))).astype(np.float32)
        q[:20] = cent[rng.integers(0, o.K, 20)]          # exactly on a centroid
        q[20:40] = 0.5 * (cent[0] + cent[1])              # halfway between two
        for nprobe in sorted({1, 3, min(o.K, 8), o.K}):
            cids, sq = idx.debug_probe(q, nprobe)
            for i in range(0, n, 97):
                c_o, s_o = o.probe(q[i], nprobe)
                assert (cids[i] == c_o).all(), (name, nprobe, i)
                assert (bits(sq[i]) == bits(s_o)).all()
        idx.free()
        o.close()
