"""Generate the golden fixtures in tests/golden/ from the reference itself.

Each case is a small seeded dataset whose index is built by the reference's
unmodified create_index (src/create_index.cpp, compiled by oracle/Makefile
with the shim) and whose search outputs are dumped by the reference's own
code through oracle/ref_harness.cpp:

  <case>.index  the index file exactly as IVF::save wrote it
  <case>.npz    rotated queries and, per query, the probe list
                (FlatInitializer::centroids_distances), per probed cluster the
                prepared query (unit_q, qq, delta, sumq from
                HASearcher::preparing), the per-lane FastScan estimates ipq and
                lower-bound masks (accumulate_one_block_high_acc at a fixed
                threshold), EX-bit inner products (IP_FUNC), the sequence of
                refined candidates, and the final ids and distances of IVF::search

Usage (needs the reference sources and `make -C oracle REF=<reference checkout>`):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "extended-rabitq_b200"))

from erq_b200 import datasets, vecs  # noqa: E402
from oracle import Reference  # noqa: E402

CREATE_INDEX = os.path.join(REPO, "oracle", "_ref", "create_index")

# name, dim, bits, n, K, queries, nprobe, k, options
CASES = [
    dict(name="d64_b3", dim=64, bits=3, n=1200, K=20, nq=10, nprobe=6, k=50),
    dict(name="d64_b4", dim=64, bits=4, n=1200, K=20, nq=10, nprobe=6, k=50),
    dict(name="d64_b5", dim=64, bits=5, n=1200, K=20, nq=10, nprobe=6, k=50),
    dict(name="d64_b7", dim=64, bits=7, n=1200, K=20, nq=10, nprobe=6, k=50),
    dict(name="d64_b8", dim=64, bits=8, n=1200, K=20, nq=10, nprobe=6, k=50),
    dict(name="d64_b9", dim=64, bits=9, n=1200, K=20, nq=10, nprobe=6, k=50),
    # DIM padded to 128, hand-made cluster sizes (empty, 1, 31, 32, 33, ...),
    # duplicated vectors, a query equal to a centroid, k larger than the
    # candidates of a single small cluster
    dict(name="d100_b8_edges", dim=100, bits=8, n=1400, K=12, nq=12, nprobe=5, k=120,
         edges=True),
    # the small 128-d Gaussian-mixture workload at reduced size (4-bit)
    dict(name="d128_b4_mix", dim=128, bits=4, n=3000, K=48, nq=12, nprobe=8, k=100),
]

EDGE_SIZES = [0, 1, 31, 32, 33, 64, 65, 96, 100, 150, 238, 590]


def build_case(c: dict, work: str) -> str:
    ds = c["name"]
    ddir = os.path.join(work, "data", ds)
    os.makedirs(ddir, exist_ok=True)
    os.makedirs(os.path.join(work, "results", "indexing_time"), exist_ok=True)
    os.makedirs(os.path.join(work, "bin"), exist_ok=True)
    seed = sum(map(ord, ds))
    base, query = datasets.gaussian_mixture(c["n"], c["dim"], 16, 0.3, seed=seed, n_query=c["nq"])
    if c.get("edges"):
        assert sum(EDGE_SIZES) == c["n"] and len(EDGE_SIZES) == c["K"]
        base[5] = base[4]          # duplicated vectors (equal distance estimates)
        base[7] = base[4]
        rng = np.random.default_rng(seed)
        order = np.argsort(base[:, 0], kind="stable")
        ids = np.empty(c["n"], np.uint32)
        pos = 0
        for cid, s in enumerate(EDGE_SIZES):
            ids[order[pos:pos + s]] = cid
            pos += s
        cent = np.zeros((c["K"], c["dim"]), np.float32)
        for cid in range(c["K"]):
            m = ids == cid
            cent[cid] = base[m].mean(axis=0) if m.any() else rng.standard_normal(c["dim"])
            # a residual of exactly zero (a singleton cluster whose centroid is
            # its member) makes the reference's fast_quantize loop for ~2^31
            # steps per dimension (max_o = 0, inc/index/Quantizer.hpp:142-196);
            # keep every member off its centroid
            cent[cid] += 0.01 * rng.standard_normal(c["dim"]).astype(np.float32)
    else:
        cent, ids = datasets.kmeans(base, c["K"], iters=10, seed=seed + 1)
    vecs.write_vecs(os.path.join(ddir, f"{ds}_base.fvecs"), base)
    vecs.write_vecs(os.path.join(ddir, f"{ds}_centroid_{c['K']}.fvecs"), cent)
    vecs.write_vecs(os.path.join(ddir, f"{ds}_cluster_id_{c['K']}.ivecs"), ids[:, None])
    subprocess.run([CREATE_INDEX, ds, str(c["K"]), str(c["bits"])], cwd=os.path.join(work, "bin"),
                   check=True, stdout=subprocess.DEVNULL, timeout=600)
    return os.path.join(ddir, f"ivf_exhaf{c['bits']}.index"), query


def dump_case(c: dict, index_path: str, query: np.ndarray) -> dict:
    r = Reference(index_path)
    qrot = r.rotate(query)
    if c.get("edges"):
        # a rotated query equal to a rotated centroid: y = 0, the unit_q fallback
        from erq_b200 import indexfile
        arr = indexfile.read_index(index_path)
        qrot[3] = arr.centroids[6]
    nq, nprobe, k, D = qrot.shape[0], c["nprobe"], c["k"], r.D
    out = dict(qrot=qrot, nprobe=np.int64(nprobe), k=np.int64(k))
    pc = np.zeros((nq, nprobe), np.uint32)
    ps = np.zeros((nq, nprobe), np.float32)
    cd = np.zeros((nq, r.K), np.float32)
    unit_q = np.zeros((nq, nprobe, D), np.float32)
    qq = np.zeros((nq, nprobe, D), np.int16)
    delta = np.zeros((nq, nprobe), np.float32)
    sumq = np.zeros((nq, nprobe), np.float32)
    shift = np.zeros((nq, nprobe), np.int32)
    ipq_all, mask_inf, mask_fin, ipq_off = [], [], [], [0]
    exip_pos, exip_val = [], []
    from erq_b200 import indexfile
    arr = indexfile.read_index(index_path)
    first_vec = arr.first_vec()
    for qi in range(nq):
        cd[qi] = r.centroid_dists(qrot[qi])
        pc[qi], ps[qi] = r.probe(qrot[qi], nprobe)
        for p in range(nprobe):
            cid = int(pc[qi, p])
            prep = r.prepare(qrot[qi], cid, ps[qi, p])
            unit_q[qi, p], qq[qi, p] = prep["unit_q"], prep["qq"]
            delta[qi, p], sumq[qi, p], shift[qi, p] = prep["delta"], prep["sumq"], prep["shift"]
            nb = (int(arr.sizes[cid]) + 31) // 32
            ipq, m1 = r.scan_cluster(qrot[qi], cid, ps[qi, p], np.float32(np.inf), nb)
            _, m2 = r.scan_cluster(qrot[qi], cid, ps[qi, p], np.float32(ps[qi, p] * 1.25), nb)
            ipq_all.append(ipq)
            mask_inf.append(m1)
            mask_fin.append(m2)
            ipq_off.append(ipq_off[-1] + ipq.size)
            for v in range(min(3, int(arr.sizes[cid]))):
                pos = int(first_vec[cid]) + v
                exip_pos.append((qi, p, pos))
                exip_val.append(r.ex_ip(prep["unit_q"], pos))
    ids, dists = r.search_dists(qrot, k, nprobe)
    ids_direct = r.search(qrot, k, nprobe)
    assert (ids == ids_direct).all(), "step-through differs from IVF::search"
    tr_ids, tr_d, tr_off = [], [], [0]
    for qi in range(nq):
        a, b = r.trace(qrot[qi], k, nprobe)
        tr_ids.append(a)
        tr_d.append(b)
        tr_off.append(tr_off[-1] + a.size)
    out.update(
        centroid_dists=cd, probe_cids=pc, probe_sqy=ps, unit_q=unit_q, qq=qq, delta=delta,
        sumq=sumq, shift=shift, ipq=np.concatenate(ipq_all) if ipq_all else np.zeros(0, np.float32),
        ipq_off=np.array(ipq_off, np.int64),
        mask_inf=np.concatenate(mask_inf) if mask_inf else np.zeros(0, np.uint32),
        mask_fin=np.concatenate(mask_fin) if mask_fin else np.zeros(0, np.uint32),
        exip_pos=np.array(exip_pos, np.int64).reshape(-1, 3),
        exip_val=np.array(exip_val, np.float32),
        ids=ids, dists=dists, trace_ids=np.concatenate(tr_ids), trace_dists=np.concatenate(tr_d),
        trace_off=np.array(tr_off, np.int64))
    r.close()
    return out


def main():
    if not os.path.exists(CREATE_INDEX):
        sys.exit("oracle/_ref/create_index missing: run `make -C oracle ref`")
    for c in CASES:
        work = tempfile.mkdtemp(prefix="erq_golden_")
        try:
            idx, query = build_case(c, work)
            data = dump_case(c, idx, query)
            shutil.copyfile(idx, os.path.join(HERE, c["name"] + ".index"))
            np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), **data)
            print(f"{c['name']}: index {os.path.getsize(idx)} B, "
                  f"trace {data['trace_ids'].size} candidates")
        finally:
            shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
