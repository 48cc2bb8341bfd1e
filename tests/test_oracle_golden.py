"""The C oracle (oracle/erq_oracle.c) against the reference's own outputs.

The golden fixtures were produced by the reference's search code
(tests/golden/make_golden.py).  Every stage must agree bit for bit: probe
lists and squared centroid distances, the prepared query (unit_q, qq, delta,
sumq), per-lane FastScan estimates and lower-bound masks, EX-bit inner
products, the sequence of refined candidates, and the final ids and
distances.
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module", params=golden_cases())
def case(request, oracle_mod):
    g = load_golden(request.param)
    o = oracle_mod.Oracle(g["path"])
    yield g, o
    o.close()


def test_centroid_distances_and_probe(case):
    g, o = case
    cent = o.centroids()
    nprobe = int(g["nprobe"])
    for qi, q in enumerate(g["qrot"]):
        d = np.array([o.lib().orc_l2sqr16(np.ascontiguousarray(q), np.ascontiguousarray(c), o.D)
                      for c in cent], np.float32)
        assert (bits(d) == bits(g["centroid_dists"][qi])).all()
        cids, sq = o.probe(q, nprobe)
        assert (cids == g["probe_cids"][qi]).all()
        assert (bits(sq) == bits(g["probe_sqy"][qi])).all()


def test_prepare(case):
    g, o = case
    cent = o.centroids()
    for qi, q in enumerate(g["qrot"]):
        for p, cid in enumerate(g["probe_cids"][qi]):
            r = o.prepare(q, cent[cid], g["probe_sqy"][qi, p])
            assert (bits(r["unit_q"]) == bits(g["unit_q"][qi, p])).all()
            assert (r["qq"] == g["qq"][qi, p]).all()
            assert bits(r["delta"]) == bits(g["delta"][qi, p])
            assert bits(r["sumq"]) == bits(g["sumq"][qi, p])
            # table entry e of group j is the subset sum of qq over e's bits
            qq = r["qq"].astype(np.int32).reshape(-1, 4)
            e = np.arange(16)
            w = np.stack([(e >> 3) & 1, (e >> 2) & 1, (e >> 1) & 1, e & 1], axis=1)
            assert (r["lut"].reshape(-1, 16) == qq @ w.T).all()


def test_scan_estimates_and_masks(case):
    g, o = case
    sizes = o.cluster_sizes()
    k = 0
    for qi, q in enumerate(g["qrot"]):
        for p, cid in enumerate(g["probe_cids"][qi]):
            sq = g["probe_sqy"][qi, p]
            lo, hi = g["ipq_off"][k], g["ipq_off"][k + 1]
            nb = (int(sizes[cid]) + 31) // 32
            mb0 = sum((g["ipq_off"][i + 1] - g["ipq_off"][i]) // 32 for i in range(k))
            S, ipq, m_inf = o.scan_cluster(q, int(cid), sq, np.float32(np.inf))
            _, _, m_fin = o.scan_cluster(q, int(cid), sq, np.float32(sq * 1.25))
            n = int(sizes[cid])
            lane_ok = (np.arange(32 * nb) < n)
            assert (bits(ipq)[lane_ok] == bits(g["ipq"][lo:hi])[lane_ok]).all()
            valid = np.array([0xFFFFFFFF if n - 32 * b >= 32 else (1 << (n - 32 * b)) - 1
                              for b in range(nb)], np.uint64).astype(np.uint32)
            assert ((m_inf & valid) == (g["mask_inf"][mb0:mb0 + nb] & valid)).all()
            assert ((m_fin & valid) == (g["mask_fin"][mb0:mb0 + nb] & valid)).all()
            # the float estimate is float(S) * delta
            assert (bits(np.float32(S.astype(np.float32) * g["delta"][qi, p]))[lane_ok]
                    == bits(ipq)[lane_ok]).all()
            k += 1


def test_ex_inner_products(case):
    g, o = case
    for (qi, p, pos), val in zip(g["exip_pos"], g["exip_val"]):
        got = o.ex_ip(g["unit_q"][qi, p], int(pos))
        assert bits(got) == bits(val)


def test_search_ids_and_distances(case):
    g, o = case
    ids, d = o.search(g["qrot"], int(g["k"]), int(g["nprobe"]))
    assert (ids == g["ids"]).all()
    assert (bits(d) == bits(g["dists"])).all()


def test_candidate_sequence(case):
    g, o = case
    for qi, q in enumerate(g["qrot"]):
        lo, hi = g["trace_off"][qi], g["trace_off"][qi + 1]
        ids, d = o.trace(q, int(g["k"]), int(g["nprobe"]))
        assert ids.size == hi - lo
        assert (ids == g["trace_ids"][lo:hi]).all()
        assert (bits(d) == bits(g["trace_dists"][lo:hi])).all()


def test_threaded_batch_matches_serial(case):
    g, o = case
    a, da = o.search(g["qrot"], int(g["k"]), int(g["nprobe"]), nthreads=1)
    b, db = o.search(g["qrot"], int(g["k"]), int(g["nprobe"]), nthreads=4)
    assert (a == b).all() and (bits(da) == bits(db)).all()
