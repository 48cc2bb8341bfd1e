#!/usr/bin/env python3
"""Benchmark of the B200 IVF search against the reference's CPU search.

Metric: queries per second of IVF::search at the smallest nprobe whose
recall@100 (against float64 brute force) reaches 0.95, on the 1M x 1536
8-bit workload (K = 4096 clusters, 10,000 queries per step, top-100).

One step = one pass of the whole query batch through rotation + coarse probe
+ FastScan scan + refinement + top-k.  `value` times steps whose raw queries
are already in device memory; `e2e` times the same steps through the C ABI
with pinned host buffers (host->device copy of the queries and
device->host copy of ids and distances inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one process per GPU (torchrun); each rank searches its own copy of
the query batch against its own replica of the index (no data-path
collective; weak scaling); time is the max over ranks.  `--impl reference`
times the reference's own CPU search (built from its sources by
oracle/Makefile) on this host's cores on samples of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import threading
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "extended-rabitq_b200")
ORACLE_DIR = os.path.join(REPO, "oracle")
for _p in (PKG, ORACLE_DIR):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

MODE_NAMES = {"plain": "plain per-query", "batched": "batched plain (plan)",
              "learned": "batched learned-probe (plan)"}
METRIC = "QPS @ recall@100≥0.95, 1M×1536 8-bit: learned-probe vs plain GPU vs ref CPU"

CONFIGS = {
    # the headline workload: openai1536-shaped synthetic data
    "sphere1536-1M-8bit": dict(
        gen="sphere", n=1_000_000, dim=1536, comps=4096, sigma=0.05, zipf=None, K=4096,
        bits=8, nq=10_000, k=100, seed=20241, nprobe=None, recall_target=0.95,
        train_queries=200_000,
        data="synthetic: seeded 4096-component unit-sphere mixture, tangent sigma 0.05, "
             "1M base + 10k queries (+200k training queries for the probe model), d=1536 "
             "(openai1536 stand-in)"),
    # batched search over very uneven clusters: Zipf(1.1) component weights
    "zipf1536-2M-7bit": dict(
        gen="sphere", n=2_000_000, dim=1536, comps=4096, sigma=0.05, zipf=1.1, K=4096,
        bits=7, nq=8192, k=100, seed=20242, nprobe=None, recall_target=0.95,
        train_queries=40_000, save_base=False, latency_batches=(1, 64, 1024, 8192),
        data="synthetic: seeded 4096-component unit-sphere mixture with Zipf(1.1) component "
             "weights, tangent sigma 0.05, 2M base + 8192 queries (+40k training queries for "
             "the probe model), d=1536"),
    # the headline data at 4 bits (EX = 3)
    "sphere1536-1M-4bit": dict(
        gen="sphere", n=1_000_000, dim=1536, comps=4096, sigma=0.05, zipf=None, K=4096,
        bits=4, nq=10_000, k=100, seed=20241, nprobe=None, recall_target=0.95,
        train_queries=0, save_base=False,
        data="synthetic: the 1M x 1536 unit-sphere mixture of the headline workload, 4-bit"),
    # learned probing + batching at scale: 10M x 768, Zipf clusters, 3/5/9 bits
    "zipf768-10M": dict(
        gen="gauss", n=10_000_000, dim=768, comps=16384, sigma=0.3, zipf=1.1, K=16384,
        bits_list=(3, 5, 9), nq=2000, k=100, seed=20245, recall_target=0.95,
        qps_queries=100_000, train_queries=10_000, max_batch=4096, c5=True,
        data="synthetic: seeded 16384-component Gaussian mixture (centres N(0, I), sigma 0.3) "
             "with Zipf(1.1) component weights, 10M base, d=768, clustered by erq_kmeans; "
             "recall on 2000 queries "
             "(exact top-100 by a TF32 shortlist of 1024 re-ranked in float64), QPS on up to "
             "100k queries in batches of sizes drawn from 1..4096 (a prefix of at least 8,192 "
             "at deep probes); probe models trained on 10k further queries"),
    # the small CPU-runnable case
    "gauss128-100k-4bit": dict(
        gen="gauss", n=100_000, dim=128, comps=256, sigma=0.3, zipf=None, K=1024,
        bits=4, nq=1000, k=100, seed=11, nprobe=None, recall_target=0.95,
        train_queries=20_000,
        data="synthetic: seeded 256-component Gaussian mixture, sigma 0.3, 100k base + 1k "
             "queries, d=128"),
}
DEFAULT_CONFIG = "sphere1536-1M-8bit"
NPROBE_SWEEP = [1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160,
                192, 256, 320, 384, 512, 768, 1024]


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ data prep
def cache_dir(name, cfg):
    key = (f"{name}-{cfg['n']}-{cfg['dim']}-{cfg['K']}-{cfg['bits']}-{cfg['nq']}-{cfg['seed']}"
           f"-{cfg.get('train_queries', 0)}")
    return os.path.join(os.environ.get("ERQ_BENCH_CACHE", "/tmp/erq_bench"), key)


def prepare(name, cfg, device="cuda"):
    """Generate data, cluster, build the index file and the ground truth on
    the GPU (torch plumbing; none of this is timed).  Cached on disk."""
    d = cache_dir(name, cfg)
    done = os.path.join(d, "done")
    if os.path.exists(done):
        return d
    import torch

    from erq_b200 import build_index, datasets, indexfile

    os.makedirs(d, exist_ok=True)
    t0 = time.time()
    nq_all = cfg["nq"] + cfg.get("train_queries", 0)
    if cfg["gen"] == "sphere":
        base, query = datasets.sphere_mixture_torch(cfg["n"], cfg["dim"], cfg["comps"],
                                                    cfg["sigma"], cfg["seed"], nq_all,
                                                    cfg["zipf"], device=device)
    else:
        base, query = datasets.gaussian_mixture_torch(cfg["n"], cfg["dim"], cfg["comps"],
                                                      cfg["sigma"], cfg["seed"], nq_all,
                                                      device=device)
    train_q = query[cfg["nq"]:]
    query = query[:cfg["nq"]]
    np.save(os.path.join(d, "train_query.npy"), train_q.cpu().numpy())
    del train_q
    log(f"generated {cfg['n']}x{cfg['dim']} in {time.time() - t0:.1f}s")
    cent, ids = datasets.kmeans_torch(base, cfg["K"], iters=20, seed=cfg["seed"] + 1)
    log(f"k-means K={cfg['K']} done at {time.time() - t0:.1f}s")
    arr = build_index.build_index_torch(base, cent, ids, cfg["bits"], seed=cfg["seed"] + 2)
    indexfile.write_index(os.path.join(d, "ivf.index"), arr)
    del arr
    log(f"index built at {time.time() - t0:.1f}s")
    gt, gtd = datasets.ground_truth_torch(base, query, cfg["k"])
    np.save(os.path.join(d, "query.npy"), query.cpu().numpy())
    np.save(os.path.join(d, "gt.npy"), gt.cpu().numpy().astype(np.uint32))
    np.save(os.path.join(d, "gt_dist.npy"), gtd.cpu().numpy())
    # the base for the distance-ratio metric on a query subset
    if cfg.get("save_base", True):
        np.save(os.path.join(d, "base.npy"), base.cpu().numpy())
    log(f"ground truth done at {time.time() - t0:.1f}s")
    del base, query, cent, ids, gt, gtd
    torch.cuda.empty_cache()
    open(done, "w").write("ok\n")
    return d


# ------------------------------------------------------------------ clocks
CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


class ClockSampler:
    """nvidia-smi samples every 100 ms on a reader thread; only samples taken
    between mark_start() and mark_end() (the timed region) are summarised."""

    def __init__(self, gpu_index: int):
        self.proc = None
        self.samples = []
        self.t0 = self.t1 = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={CLOCK_FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(gpu_index), "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.first = threading.Event()
        self.reader = threading.Thread(target=self._read, daemon=True)
        self.reader.start()
        self.first.wait(timeout=10.0)

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.monotonic(), line))
            self.first.set()

    def mark_start(self):
        self.t0 = time.monotonic()

    def mark_end(self):
        self.t1 = time.monotonic()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.reader.join(timeout=5)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0 = self.t0 if self.t0 is not None else 0.0
        t1 = (self.t1 if self.t1 is not None else time.monotonic()) + 0.15
        for t, line in self.samples:
            if not (t0 <= t <= t1):
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- CPU baselines
def cpu_has_avx512() -> bool:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return False
    return all(f in flags for f in ("avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512cd"))


def cpu_searcher(index_path):
    """The reference's own search (stock flags) when it is built and the host
    has AVX-512, else the C restatement.  Returns (searcher, kind, note)."""
    import oracle

    if oracle.reference_available(stock=True) and cpu_has_avx512():
        return (oracle.Reference(index_path, stock=True), "reference",
                "reference compiled with its own -Ofast flags but -march=x86-64-v4 (AVX-512) "
                "in place of -march=native, so the binary runs on any AVX-512 host")
    note = ("reference build missing" if not oracle.reference_available(stock=True)
            else "host lacks AVX-512; reference cannot run")
    oracle.build_oracle()
    return oracle.Oracle(index_path), "port", note


def time_cpu(searcher, kind, query_raw, k, nprobe, threads, budget_s, max_n):
    """Time searcher on a bounded sample: queries whose measured cost fits
    budget_s.  Returns (qps, n, seconds, rotate_s, search_s)."""
    if kind == "reference":
        rotate = searcher.rotate
    else:
        P = searcher.rotation()
        D = P.shape[0]

        def rotate(q):
            pad = np.zeros((q.shape[0], D), np.float32)
            pad[:, :q.shape[1]] = q
            return pad @ P
    probe_n = min(max_n, max(threads * 4, 32))
    q = query_raw[:probe_n]
    t0 = time.perf_counter()
    qr = rotate(q)
    searcher.search(qr, k, nprobe, nthreads=threads)
    per_q = (time.perf_counter() - t0) / probe_n
    n = int(min(max_n, max(probe_n, budget_s / max(per_q, 1e-9))))
    q = query_raw[:n]
    t0 = time.perf_counter()
    qr = rotate(q)
    t1 = time.perf_counter()
    searcher.search(qr, k, nprobe, nthreads=threads)
    t2 = time.perf_counter()
    return n / (t2 - t0), n, t2 - t0, t1 - t0, t2 - t1


PARITY_QUERIES = 200
# A query whose most likely probe depth has a probability below this falls
# back to the fixed nprobe (8 depths: a uniform guess gives each 0.125).
LEARNED_MIN_PROB = 0.25

# DRAM bytes (read + write) per algorithmic byte, from one-pass ncu captures of
# dram__bytes_read.sum + dram__bytes_write.sum on this bench's headline
# workload, per mode and kernel (profiles/dram_traffic_sphere1536_1M_8bit.md);
# a launch's traffic is that ratio times its algorithmic bytes.  The ratios
# hold for the headline workload, not for other configurations.
DRAM_PER_ALGORITHMIC_BYTE = {
    ("plain", "scan_kernel"): 0.0589, ("plain", "refine_kernel"): 0.397,
    ("batched", "scan_batched_kernel"): 0.0587, ("batched", "refine_kernel"): 0.397,
    ("learned", "scan_batched_kernel"): 0.260, ("learned", "refine_kernel"): 0.397,
}


def json_peak():
    """hbm_gbs of MEASURED_PEAKS.json, or None when the file is absent."""
    try:
        return json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        return None


def traffic_per_launch(mode, kernel, step_bytes, launches_per_step):
    r = DRAM_PER_ALGORITHMIC_BYTE.get((mode, kernel))
    if r is None or not launches_per_step:
        return None
    return int(r * step_bytes / launches_per_step)


def reference_parity(index_path, idx, query, k, nprobe, model=None, confidence=None):
    """Results of the GPU search on the first PARITY_QUERIES queries against the
    reference's own IVF::search (strict IEEE build) on the same index file and
    the same rotated-query bytes: the plain search at `nprobe`, and with a
    probe model the learned search query by query at the depth it chose.
    Outside every timed region."""
    import oracle

    from erq_b200 import learned

    if oracle.reference_available():
        ref, kind = oracle.Reference(index_path), "reference IVF::search, strict IEEE build"

        def ref_search(q, kk, npb):
            return ref.search_dists(q, kk, npb)
    else:
        oracle.build_oracle()
        ref, kind = oracle.Oracle(index_path), "C restatement (reference build missing)"

        def ref_search(q, kk, npb):
            return ref.search(q, kk, npb, nthreads=os.cpu_count() or 1)
    qrot = idx.rotate(query[:PARITY_QUERIES])
    out = {"queries": int(qrot.shape[0]), "against": kind}

    def compare(ids, d, depth):
        ids_eq = dist_eq = True
        for u in np.unique(depth):
            sel = np.flatnonzero(depth == u)
            ri, rd = ref_search(qrot[sel], k, int(u))
            ids_eq &= bool((ids[sel] == ri).all())
            dist_eq &= bool((d[sel].view(np.uint32) == rd.view(np.uint32)).all())
        return {"ids_equal": ids_eq, "dist_bits_equal": dist_eq}

    ids, d = idx.search_batch(qrot, k, nprobe)
    out["plain"] = dict(nprobe=nprobe, **compare(ids, d, np.full(qrot.shape[0], nprobe)))
    if model is not None:
        ids, d, used = learned.search_learned(idx, model, qrot, k, nprobe_fallback=nprobe,
                                              confidence=confidence, min_prob=LEARNED_MIN_PROB)
        out["learned"] = dict(mean_nprobe=round(float(used.mean()), 3), **compare(ids, d, used))
    ref.close()
    return out


# ------------------------------------------------------------------ helpers
from erq_b200.replicas import barrier, finish as dist_finish, max_over_ranks  # noqa: E402


def dist_setup(args):
    from erq_b200 import replicas

    return replicas.init(timeout_s=600)


def choose_nprobe(idx, qraw, gt, cfg):
    """Smallest nprobe of the sweep reaching the recall target (all queries)."""
    from erq_b200 import metrics

    k = cfg["k"]
    sweep = [p for p in NPROBE_SWEEP if p <= cfg["K"]]
    if cfg.get("nprobe"):
        sweep = [cfg["nprobe"]] + [p for p in sweep if p > cfg["nprobe"]]
    best = None
    for p in sweep:
        ids, _ = idx.search_raw(qraw, k, p, with_dists=False)
        r = metrics.recall_at_k(ids.view(np.uint32) if ids.dtype != np.uint32 else ids, gt, k)
        log(f"nprobe={p}: recall@{k}={r:.4f}")
        best = (p, r, ids)
        if r >= cfg["recall_target"]:
            break
    return best


def timed(step, steps, warmup, world, stream, clock_gpu=None, label=None):
    """`warmup` untimed calls, then `steps` calls between CUDA events on
    `stream` bracketed by barrier + synchronize; returns (max-over-ranks ms,
    per-kernel profile of the timed calls, clock samples).  `label` names an
    NVTX range around the timed calls (for a profiler's range filter)."""
    import torch

    from erq_b200 import _lib as L

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(clock_gpu) if clock_gpu is not None else None
    L.profile_reset()
    L.profile_enable(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if sampler:
        sampler.mark_start()
    if label:
        torch.cuda.nvtx.range_push(label)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    if label:
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if sampler:
        sampler.mark_end()
    L.profile_enable(False)
    barrier(world)
    clocks = sampler.stop() if sampler else None
    prof = L.profile_read()
    return max_over_ranks(e0.elapsed_time(e1), world), prof, clocks


def learned_model(idx, d, cfg, plain_nprobe, train=None):
    """The probe model of this workload, trained once and cached: labels from
    the plain search on the training queries, features from the probe kernel,
    training on the GPU by the library's kernels."""
    from erq_b200 import learned

    bins = learned.scaled_bins(plain_nprobe, cfg["K"])
    path = os.path.join(d, f"probe-b{cfg['bits']}-" + "-".join(map(str, bins)) + ".model")
    if os.path.exists(path):
        return learned.ProbeModel.load(path), json.load(open(path + ".json"))
    t0 = time.time()
    train_q = np.load(os.path.join(d, "train_query.npy")) if train is None else train
    rot = idx.rotate(train_q)
    del train_q
    labels = learned.make_labels(idx, rot, cfg["k"], bins)
    # exhaustive probing reads the whole index per query: fewer queries for
    # the 10M-vector index
    n_agree = 1000 if cfg["n"] <= 2_000_000 else 200
    agree = learned.exhaustive_agreement(idx, rot[:n_agree], cfg["k"], bins[-1])
    feats = learned.probe_features(idx, rot)
    del rot
    model = learned.ProbeModel.train(feats, labels, bins, epochs=8, batch=1024, lr=1e-3,
                                     seed=cfg["seed"] + 3)
    hist = np.bincount(labels, minlength=len(bins)).tolist()
    meta = {"train_queries": int(labels.size), "label_hist": hist, "bins": list(bins),
            "labels": f"smallest depth whose top-{cfg['k']} set equals that at the deepest "
                      f"bin ({bins[-1]} probes)",
            "deepest_bin_equals_exhaustive": round(agree, 4),
            "exhaustive_sample": n_agree,
            "final_loss": round(model.final_loss, 4), "train_s": round(time.time() - t0, 1)}
    model.save(path)
    json.dump(meta, open(path + ".json", "w"))
    log(f"probe model: {meta}")
    return model, meta


# ------------------------------------------------------------------ our arm
def run_ours(args, cfg, name):
    import torch

    from erq_b200 import IVF, indexfile, learned, metrics

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if rank == 0:
        d = prepare(name, cfg)
    barrier(world)
    d = prepare(name, cfg) if rank != 0 else d
    index_path = os.path.join(d, "ivf.index")
    query = np.load(os.path.join(d, "query.npy"))
    gt = np.load(os.path.join(d, "gt.npy"))
    if args.queries:
        query, gt = query[:args.queries], gt[:args.queries]
    nq, k = query.shape[0], cfg["k"]
    target = cfg["recall_target"]

    idx = IVF(index_path, device=local)
    if args.nprobe:
        cfg = dict(cfg, nprobe=args.nprobe)
    nprobe, recall, ids0 = choose_nprobe(idx, query, gt, cfg)
    from erq_b200 import _lib as L

    L.probe_fallbacks(local, reset=True)
    L.refine_stats(local, enable=True)
    idx.search_raw(query, k, nprobe, with_dists=False)
    rst_plain = L.refine_stats(local, enable=False)
    cand_plain = rst_plain["candidates"]
    fallback_rate = L.probe_fallbacks(local, reset=True) / nq
    log(f"probe fallback rate {fallback_rate:.5f}; refinement per query: "
        + ", ".join(f"{kk} {v / nq:.1f}" for kk, v in rst_plain.items()))
    base = np.load(os.path.join(d, "base.npy"), mmap_mode="r")
    sub = min(1000, nq)
    arr = indexfile.read_index(index_path)
    nblocks = (arr.sizes.astype(np.int64) + 31) // 32
    block_bytes = 4 * arr.D + 128
    cand_bytes = arr.D * arr.EX // 8 + 8  # EX-code row + xipnorm + id per exact candidate
    qrot_h = idx.rotate(query)
    cids, _ = idx.debug_probe(qrot_h, max(nprobe, learned.scaled_bins(nprobe, arr.K)[-1]))
    del arr

    stream = torch.cuda.current_stream()
    qd = torch.from_numpy(query).cuda()
    ids_d = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dist_d = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    qh = torch.from_numpy(query).pin_memory()
    ids_h = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    dist_h = torch.empty((nq, k), dtype=torch.float32).pin_memory()

    # --- plain fixed-nprobe search
    def plain_dev():
        idx.search_raw(qd, k, nprobe, ids=ids_d, dists=dist_d, stream=stream)

    def plain_host():
        idx.search_raw(qh, k, nprobe, ids=ids_h, dists=dist_h, stream=stream)

    ms_p, prof_p, clocks_p = timed(plain_dev, args.steps, args.warmup, world, stream, local,
                                   label="plain")
    assert (ids_d.cpu().numpy().view(np.uint32) == ids0).all()
    plain = {"value": round(world * nq * args.steps / (ms_p / 1e3), 1), "nprobe": nprobe,
             "recall@100": round(recall, 5), "ms_per_step": round(ms_p / args.steps, 4),
             "refine_per_query": {kk: round(v / nq, 2) for kk, v in rst_plain.items()},
             "kernels_ms_per_step": {kk: round(v[1] / args.steps, 4) for kk, v in prof_p.items()
                                     if v[0]}}
    ms_pe = None
    if not args.no_e2e:
        ms_pe, _, _ = timed(plain_host, args.steps, args.warmup, world, stream)
        assert (ids_h.numpy().view(np.uint32) == ids0).all()
        plain["e2e"] = round(world * nq * args.steps / (ms_pe / 1e3), 1)
    scan_bytes_plain = int(nblocks[cids[:, :nprobe].astype(np.int64)].sum()) * block_bytes

    # --- batched plans (CUDA graphs, work-list scan, autotuned tiles)
    from erq_b200 import Plan

    qh2 = qh.clone().pin_memory()
    ids_h2 = torch.empty_like(ids_h).pin_memory()
    dist_h2 = torch.empty_like(dist_h).pin_memory()

    def timed_two_plans(plans, steps, warmup):
        """Pinned host buffers, two plans of the same settings on two streams,
        consecutive steps alternating between them (a serving loop with two
        batches in flight): a step's copies in and out run under the other
        plan's search.  Timed between CUDA events on `stream`, the second
        stream joined before the end event; returns max-over-ranks ms."""
        streams = (stream, torch.cuda.Stream())
        bufs = ((qh, ids_h, dist_h), (qh2, ids_h2, dist_h2))

        def step(i):
            plans[i % 2].search_buffers_async(*bufs[i % 2], stream=streams[i % 2])

        for i in range(warmup):
            step(i)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        streams[1].wait_event(e0)
        for i in range(steps):
            step(i)
        streams[0].wait_stream(streams[1])
        e1.record(streams[0])
        torch.cuda.synchronize()
        barrier(world)
        return max_over_ranks(e0.elapsed_time(e1), world)

    def twin_plan(plan, tune, mdl=None, conf=None):
        """A second plan with `plan`'s settings, for the two-stream serving loop."""
        tw = Plan(idx, max_batch=nq, k=k, nprobe=nprobe, model=mdl, raw=True)
        if mdl is not None:
            tw.set_learned(conf, LEARNED_MIN_PROB)
        tw.set_tuning(nq, tune["queries_per_item"], tune["blocks_per_item"], tune["warps"],
                      tune["refine_warps"])
        return tw

    def plan_mode(plan, expect, label, twin=None):
        def dev():
            plan.search_buffers(qd, ids_d, dist_d, stream=stream)

        def host():  # pinned host buffers, each call's copy-in under the search before
            plan.search_buffers_async(qh, ids_h, dist_h, stream=stream)

        def host_sync():  # each call returns with its results in host memory
            plan.search_buffers(qh, ids_h, dist_h, stream=stream)

        ms, _, clocks = timed(dev, args.steps, args.warmup, world, stream, local, label=label)
        assert (ids_d.cpu().numpy().view(np.uint32) == expect).all()
        e2e = None
        plan.e2e_one_stream_ms = None
        if not args.no_e2e:
            e2e, _, _ = timed(host, args.steps, args.warmup, world, stream)
            assert (ids_h.numpy().view(np.uint32) == expect).all()
            plan.e2e_one_stream_ms = e2e
            e2e_sync, _, _ = timed(host_sync, args.steps, args.warmup, world, stream)
            assert (ids_h.numpy().view(np.uint32) == expect).all()
            plan.e2e_sync_ms = e2e_sync
            if twin is not None:
                ids_h.fill_(-1)
                ids_h2.fill_(-1)
                e2e = timed_two_plans((plan, twin), args.steps, args.warmup)
                assert (ids_h.numpy().view(np.uint32) == expect).all()
                assert (ids_h2.numpy().view(np.uint32) == expect).all()
        # per-kernel times: the same steps with the kernels launched one by one
        plan.set_graphs(False)
        _, prof, _ = timed(dev, args.steps, 1, world, stream, label=label + "-kernels")
        plan.set_graphs(True)
        return ms, e2e, clocks, prof

    modes = {"plain": {"ms": ms_p, "prof": prof_p, "clocks": clocks_p, "recall": recall,
                       "ids": ids0, "scan_bytes": scan_bytes_plain, "e2e_ms": ms_pe,
                       "refine_bytes": cand_plain * cand_bytes}}
    batched = None
    if not args.no_batched:
        plan_b = Plan(idx, max_batch=nq, k=k, nprobe=nprobe, raw=True)
        tune_b, _ = plan_b.autotune(query, reps=2)
        twin_b = None if args.no_e2e else twin_plan(plan_b, tune_b)
        ms_b, e2e_b, clocks_b, prof_b = plan_mode(plan_b, ids0, "batched", twin_b)
        batched = {"value": round(world * nq * args.steps / (ms_b / 1e3), 1), "nprobe": nprobe,
                   "recall@100": round(recall, 5), "ms_per_step": round(ms_b / args.steps, 4),
                   "tuning": tune_b,
                   "kernels_ms_per_step": {kk: round(v[1] / args.steps, 4) for kk, v in prof_b.items()
                                           if v[0]}}
        if e2e_b is not None:
            batched["e2e"] = round(world * nq * args.steps / (e2e_b / 1e3), 1)
            batched["e2e_one_stream"] = round(world * nq * args.steps / (plan_b.e2e_one_stream_ms / 1e3), 1)
            batched["e2e_sync"] = round(world * nq * args.steps / (plan_b.e2e_sync_ms / 1e3), 1)
        modes["batched"] = {"ms": ms_b, "prof": prof_b, "clocks": clocks_b, "recall": recall,
                            "ids": ids0, "scan_bytes": scan_bytes_plain, "e2e_ms": e2e_b,
                            "e2e_one_stream_ms": plan_b.e2e_one_stream_ms,
                            "refine_bytes": cand_plain * cand_bytes}
        plan_b.free()
        if twin_b is not None:
            twin_b.free()

    # --- learned per-query depth, batched
    learned_info = None
    learned_for_parity = (None, None)
    model = None
    if not args.no_learned and cfg.get("train_queries"):
        model, meta = learned_model(idx, d, cfg, nprobe)
        plan_l = Plan(idx, max_batch=nq, k=k, nprobe=nprobe, model=model, raw=True)
        best = None
        # lowest confidence first: the first that meets the recall target
        # probes the fewest clusters
        for conf in (0.005, 0.01, 0.02, 0.05, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9,
                     0.95, 0.99):
            plan_l.set_learned(conf, LEARNED_MIN_PROB)
            ids_l, _, used = plan_l.search(query, with_dists=False, with_nprobe=True)
            r = metrics.recall_at_k(ids_l, gt, k)
            log(f"learned confidence={conf}: recall@{k}={r:.4f}, mean nprobe "
                f"{used.mean():.3f}")
            if r >= target:
                best = (conf, r, ids_l, used)
                break
        if best is not None:
            conf, r_l, ids_l, used = best
            plan_l.set_learned(conf, LEARNED_MIN_PROB)
            model_fallback = learned.fallback_rate(model, learned.probe_features(idx, qrot_h),
                                                   LEARNED_MIN_PROB)
            L.probe_fallbacks(local, reset=True)
            plan_l.set_graphs(False)  # counting is fixed into a graph when it is captured
            L.refine_stats(local, enable=True)
            plan_l.search(query, with_dists=False)
            rst_l = L.refine_stats(local, enable=False)
            cand_l = rst_l["candidates"]
            plan_l.set_graphs(True)
            learned_fallback_rate = L.probe_fallbacks(local, reset=True) / nq
            log(f"learned probe fallback rate {learned_fallback_rate:.5f}; refinement per "
                "query: " + ", ".join(f"{kk} {v / nq:.1f}" for kk, v in rst_l.items()))
            tune_l, _ = plan_l.autotune(query, reps=2)
            twin_l = None if args.no_e2e else twin_plan(plan_l, tune_l, model, conf)
            ms_l, e2e_l, clocks_l, prof_l = plan_mode(plan_l, ids_l, "learned", twin_l)
            if twin_l is not None:
                twin_l.free()
            take = np.arange(cids.shape[1])[None, :] < used.astype(np.int64)[:, None]
            scan_bytes_l = int(nblocks[cids.astype(np.int64)][take].sum()) * block_bytes
            learned_info = {"value": round(world * nq * args.steps / (ms_l / 1e3), 1),
                            "confidence": conf, "mean_nprobe": round(float(used.mean()), 4),
                            "recall@100": round(r_l, 5),
                            "ms_per_step": round(ms_l / args.steps, 4), "tuning": tune_l,
                            "min_prob": LEARNED_MIN_PROB,
                            "model_fallback_rate": round(model_fallback, 5),
                            "exact_probe_fallback_rate": round(learned_fallback_rate, 5),
                            "refine_per_query": {kk: round(v / nq, 2) for kk, v in rst_l.items()},
                            "kernels_ms_per_step": {kk: round(v[1] / args.steps, 4)
                                                    for kk, v in prof_l.items() if v[0]},
                            "model": meta}
            if e2e_l is not None:
                learned_info["e2e"] = round(world * nq * args.steps / (e2e_l / 1e3), 1)
                learned_info["e2e_one_stream"] = round(
                    world * nq * args.steps / (plan_l.e2e_one_stream_ms / 1e3), 1)
                learned_info["e2e_sync"] = round(world * nq * args.steps / (plan_l.e2e_sync_ms / 1e3), 1)
            modes["learned"] = {"ms": ms_l, "prof": prof_l, "clocks": clocks_l, "recall": r_l,
                                "ids": ids_l, "scan_bytes": scan_bytes_l, "e2e_ms": e2e_l,
                                "e2e_one_stream_ms": plan_l.e2e_one_stream_ms,
                                "refine_bytes": cand_l * cand_bytes}
            learned_for_parity = (model, conf)
        plan_l.free()
    mode = min(modes, key=lambda m: modes[m]["ms"])
    chosen = modes[mode]

    # the scan at deeper probes (scan-dominated points of the plain path;
    # not the headline, whose nprobe is the smallest reaching the target)
    depth_sweep = []
    if not args.no_depth_sweep:
        nd = min(nq, 2000)
        qd_s = qd[:nd]
        ids_s = torch.empty((nd, k), dtype=torch.int32, device="cuda")
        cids_d, _ = idx.debug_probe(qrot_h[:nd], 64)
        for npd in (16, 64):
            def depth_step():
                idx.search_raw(qd_s, k, npd, ids=ids_s, with_dists=False, stream=stream)

            ms_d, prof_d, _ = timed(depth_step, 5, 3, world, stream)
            nl, tms = prof_d.get("scan", (0, 0.0))
            sbytes = int(nblocks[cids_d[:, :npd].astype(np.int64)].sum()) * block_bytes
            ach = sbytes * 5 / (tms / 1e3) / 1e9 if tms else 0.0
            depth_sweep.append({"nprobe": npd, "queries": nd, "kernel": "scan_kernel",
                                "scan_ms_per_step": round(tms / 5, 4),
                                "scan_bytes_per_step": sbytes, "achieved_gbs": round(ach, 1),
                                "frac": round(ach / (json_peak() or 6650.0), 4),
                                "refine_ms_per_step": round(prof_d.get("refine", (0, 0.0))[1] / 5, 4),
                                "ms_per_step": round(ms_d / 5, 4)})
            log(f"scan depth sweep: {depth_sweep[-1]}")

    ratio = metrics.average_distance_ratio(query[:sub], base, chosen["ids"][:sub].astype(np.int64),
                                           gt[:sub].astype(np.int64), k)
    prof = chosen["prof"]
    launches = sum(v[0] for v in prof.values())
    peak = json_peak()
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    # algorithmic bytes per step of the two HBM-side kernels: scan = the
    # probed clusters' code blocks (4D + 128 B per block), refine = the exact
    # candidates' EX-code rows + xipnorm + id (D*EX/8 + 8 B each)
    headline = name == DEFAULT_CONFIG and not args.queries and not args.nprobe

    def mode_rooflines(m):
        md = modes[m]
        names = {"scan": "scan_kernel" if m == "plain" else "scan_batched_kernel",
                 "refine": "refine_kernel"}
        res = {}
        for kn, step_bytes in (("scan", md["scan_bytes"]), ("refine", md["refine_bytes"])):
            n_launch, tot_ms = md["prof"].get(kn, (0, 0.0))
            if not n_launch:
                continue
            achieved = step_bytes * args.steps / n_launch / (tot_ms / n_launch / 1e3) / 1e9
            res[kn] = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                       "unit": "GB/s", "frac": round(achieved / peak, 4),
                       "traffic": (traffic_per_launch(m, names[kn], step_bytes, n_launch / args.steps)
                                   if headline else None),
                       "kernel": names[kn], "ms_per_step": round(tot_ms / args.steps, 4),
                       "bytes_per_step": int(step_bytes),
                       "peak_source": f"{peak_src} hbm_gbs (copy)"}
        return res

    rooflines = mode_rooflines(mode)
    for m, info in (("plain", plain), ("batched", batched), ("learned", learned_info)):
        if info is not None and m in modes:
            info["rooflines"] = mode_rooflines(m)
    dominant = max(rooflines, key=lambda kn: rooflines[kn]["ms_per_step"]) if rooflines else None
    e2e_ms = chosen["e2e_ms"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        searcher, kind, note = cpu_searcher(index_path)
        threads = os.cpu_count() or 1
        qps, n, sec, rot_s, srch_s = time_cpu(searcher, kind, query, k, nprobe, threads,
                                              args.cpu_budget, nq)
        cpu = {"value": round(qps, 2), "unit": "queries/s", "cores": threads, "kind": kind,
               "sample": f"first {n} of the {nq} queries at nprobe={nprobe}, "
                         f"{threads} threads, {sec:.1f}s (rotate {rot_s:.2f}s + search "
                         f"{srch_s:.2f}s)" + (f"; {note}" if note else "")}
        searcher.close()
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        parity = reference_parity(index_path, idx, query, k, nprobe, *learned_for_parity)
        log(f"parity sample: {parity}")
    if model is not None:
        model.free()
    if rank == 0:
        ms = chosen["ms"]
        out = {
            "metric": METRIC, "value": round(world * nq * args.steps / (ms / 1e3), 1),
            "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": cfg["data"],
            "config": {"workload": f"{name}: {MODE_NAMES[mode]} "
                                   f"GPU search, {cfg['n']}x{cfg['dim']}, K={cfg['K']}, "
                                   f"{cfg['bits']}-bit, {nq} queries per step, top-{k}",
                       "mode": mode, "nprobe": nprobe, "recall@100": round(chosen["recall"], 5),
                       "distance_ratio": round(ratio, 5), "queries_per_step": nq,
                       "exact_probe_fallback_rate": round(fallback_rate, 5),
                       "parallelism": f"replicas x{world} (queries replicated per GPU)",
                       "l2": "inputs larger than L2: every step streams "
                             f"{chosen['scan_bytes'] / 1e9:.1f} GB of packed codes from a "
                             f"{os.path.getsize(index_path) / 1e9:.2f} GB index"},
            "plain_gpu": plain,
            "batched_gpu": batched,
            "learned_gpu": learned_info,
            "e2e": None if e2e_ms is None else {
                "value": round(world * nq * args.steps / (e2e_ms / 1e3), 1), "unit": "queries/s",
                "h2d_bytes_per_step": int(nq * query.shape[1] * 4),
                "d2h_bytes_per_step": int(nq * k * 8),
                "api": ("erq_search_raw, pinned host buffers, one synchronous call per step"
                        if mode == "plain" else
                        "erq_plan_search_async on two plans of the same settings and two "
                        "streams, consecutive steps alternating, pinned host buffers: a step's "
                        "copies in and out run under the other plan's search; queries copied in "
                        "and results copied out every step"),
                "one_stream": (None if chosen.get("e2e_one_stream_ms") is None else round(
                    world * nq * args.steps / (chosen["e2e_one_stream_ms"] / 1e3), 1))},
            "gpu_launches": int(launches),
            "roofline": rooflines.get(dominant),
            "roofline_other": {kn: r for kn, r in rooflines.items() if kn != dominant},
            "scan_depth_sweep": depth_sweep,
            "kernels_ms_per_step": {kk: round(v[1] / args.steps, 4) for kk, v in prof.items()
                                    if v[0]},
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": chosen["clocks"],
        }
    idx.free()
    dist_finish(world)
    return out if rank == 0 else None


# ------------------------------------------------- secondary workloads
def _timed_calls(fn, calls, warmup):
    """Per-call device times (ms) of fn() on the current stream."""
    import torch

    for _ in range(warmup):
        fn()
    st = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(calls)]
    torch.cuda.synchronize()
    for c in range(calls):
        ev[c][0].record(st)
        fn()
        ev[c][1].record(st)
    torch.cuda.synchronize()
    return np.array([a.elapsed_time(b) for a, b in ev])


def secondary_small(args):
    """100k x 128, 4-bit, nprobe 16/32/64: one query per call (p50/p99 and
    QPS; through erq_search_raw and through a plan's replayed graph) and the
    whole 1,000-query batch per call, with recall@100."""
    import torch

    from erq_b200 import IVF, Plan, metrics

    name = "gauss128-100k-4bit"
    cfg = CONFIGS[name]
    d = prepare(name, cfg)
    idx = IVF(os.path.join(d, "ivf.index"))
    query = np.load(os.path.join(d, "query.npy"))
    gt = np.load(os.path.join(d, "gt.npy"))
    qd = torch.from_numpy(query).cuda()
    k = cfg["k"]
    ids = torch.empty((query.shape[0], k), dtype=torch.int32, device="cuda")
    dist = torch.empty((query.shape[0], k), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    out = {}
    for nprobe in (16, 32, 64):
        r_ids, _ = idx.search_raw(query, k, nprobe, with_dists=False)
        rec = metrics.recall_at_k(r_ids, gt, k)
        calls = iter(range(1 << 30))

        def one_query():
            i = next(calls) % query.shape[0]
            idx.search_raw(qd[i:i + 1], k, nprobe, ids=ids[:1], dists=dist[:1], stream=st)

        one = _timed_calls(one_query, 300, 10)
        # the same through a plan for batches of one (its CUDA graph replayed)
        plan = Plan(idx, max_batch=1, k=k, nprobe=nprobe, raw=True)

        def one_query_plan():
            i = next(calls) % query.shape[0]
            plan.search_buffers(qd[i:i + 1], ids[:1], dist[:1], stream=st)

        one_p = _timed_calls(one_query_plan, 300, 10)
        plan.free()
        batch = _timed_calls(lambda: idx.search_raw(qd, k, nprobe, ids=ids, dists=dist, stream=st),
                             20, 3)
        out[str(nprobe)] = {"recall@100": round(rec, 5),
                            "one_query_per_call": {"qps": round(1e3 / one.mean(), 1),
                                                   "p50_ms": round(float(np.percentile(one, 50)), 4),
                                                   "p99_ms": round(float(np.percentile(one, 99)), 4)},
                            "one_query_per_call_plan": {
                                "qps": round(1e3 / one_p.mean(), 1),
                                "p50_ms": round(float(np.percentile(one_p, 50)), 4),
                                "p99_ms": round(float(np.percentile(one_p, 99)), 4)},
                            "batch_1000_qps": round(1e3 * query.shape[0] / batch.mean(), 1)}
    idx.free()
    return {"workload": f"{name}: 100000x128, K=1024, 4-bit, top-100, one query per call and "
                        "1000-query batches", "nprobe": out}


def secondary_4bit(args):
    """The headline data at 4 bits: plain per-query and batched plan QPS at
    the smallest nprobe reaching recall@100 >= 0.95 (10k queries per call)."""
    import torch

    from erq_b200 import IVF, Plan

    name = "sphere1536-1M-4bit"
    cfg = CONFIGS[name]
    d = prepare(name, cfg)
    idx = IVF(os.path.join(d, "ivf.index"))
    query = np.load(os.path.join(d, "query.npy"))
    gt = np.load(os.path.join(d, "gt.npy"))
    nprobe, rec, ids0 = choose_nprobe(idx, query, gt, cfg)
    qd = torch.from_numpy(query).cuda()
    k, nq = cfg["k"], query.shape[0]
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dist = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream()
    plain = _timed_calls(lambda: idx.search_raw(qd, k, nprobe, ids=ids, dists=dist, stream=st), 10, 3)
    plan = Plan(idx, max_batch=nq, k=k, nprobe=nprobe, raw=True)
    plan.autotune(query, reps=2)
    batched = _timed_calls(lambda: plan.search_buffers(qd, ids, dist, stream=st), 10, 3)
    assert (ids.cpu().numpy().view(np.uint32) == ids0).all()
    plan.free()
    idx.free()
    return {"workload": f"{name}: 1000000x1536, K=4096, 4-bit, 10000 queries per call, top-100",
            "nprobe": nprobe, "recall@100": round(rec, 5),
            "plain_qps": round(1e3 * nq / plain.mean(), 1),
            "batched_qps": round(1e3 * nq / batched.mean(), 1)}


def secondary_zipf_learned(args):
    """Zipf 2M x 1536, 7-bit, batches of 8192: the batched plain plan at the
    smallest nprobe reaching recall@100 >= 0.95 against the batched learned
    plan at the lowest confidence reaching it (probe depths scaled to the
    workload, fallback below LEARNED_MIN_PROB)."""
    import torch

    from erq_b200 import IVF, Plan, learned, metrics

    name = "zipf1536-2M-7bit"
    cfg = CONFIGS[name]
    d = prepare(name, cfg)
    idx = IVF(os.path.join(d, "ivf.index"))
    query = np.load(os.path.join(d, "query.npy"))
    gt = np.load(os.path.join(d, "gt.npy"))
    nprobe, rec, ids0 = choose_nprobe(idx, query, gt, cfg)
    k, nq = cfg["k"], query.shape[0]
    qd = torch.from_numpy(query).cuda()
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    plan = Plan(idx, max_batch=nq, k=k, nprobe=nprobe, raw=True)
    plan.autotune(query, reps=1)
    plain = _timed_calls(lambda: plan.search_buffers(qd, ids, stream=st), 5, 3)
    plan.free()
    model, meta = learned_model(idx, d, cfg, nprobe)
    plan_l = Plan(idx, max_batch=nq, k=k, nprobe=nprobe, model=model, raw=True)
    best = None
    for conf in (0.005, 0.01, 0.02, 0.05, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 0.95, 0.99):
        plan_l.set_learned(conf, LEARNED_MIN_PROB)
        ids_l, _, used = plan_l.search(query, with_dists=False, with_nprobe=True)
        r = metrics.recall_at_k(ids_l, gt, k)
        log(f"zipf learned confidence={conf}: recall@{k}={r:.4f}, mean nprobe {used.mean():.1f}")
        if r >= cfg["recall_target"]:
            best = (conf, r, used)
            break
    res = {"workload": f"{name}: 2000000x1536, K=4096 Zipf(1.1) clusters, 7-bit, batches of "
                       f"{nq}, top-100",
           "plain": {"nprobe": nprobe, "recall@100": round(rec, 5),
                     "qps": round(1e3 * nq / plain.mean(), 1)},
           "model": meta}
    if best is not None:
        conf, r_l, used = best
        plan_l.set_learned(conf, LEARNED_MIN_PROB)
        plan_l.autotune(query, reps=1)
        lt = _timed_calls(lambda: plan_l.search_buffers(qd, ids, stream=st), 5, 3)
        feats = learned.probe_features(idx, idx.rotate(query))
        res["learned"] = {"confidence": conf, "recall@100": round(r_l, 5),
                          "mean_nprobe": round(float(used.mean()), 2),
                          "min_prob": LEARNED_MIN_PROB,
                          "model_fallback_rate": round(learned.fallback_rate(model, feats,
                                                                             LEARNED_MIN_PROB), 5),
                          "qps": round(1e3 * nq / lt.mean(), 1)}
        res["learned_over_plain"] = round(res["learned"]["qps"] / res["plain"]["qps"], 3)
    plan_l.free()
    model.free()
    idx.free()
    return res


def run_secondary(args):
    """The other workloads of the benchmark suite, each guarded: a failure is
    reported in its entry and does not touch the headline line."""
    import torch

    out = {}
    for key, fn in (("gauss128-100k-4bit", secondary_small), ("sphere1536-1M-4bit", secondary_4bit),
                    ("zipf1536-2M-7bit-learned", secondary_zipf_learned)):
        t0 = time.time()
        try:
            out[key] = fn(args)
        except Exception as e:  # noqa: BLE001 - recorded, the headline stands
            out[key] = {"error": f"{type(e).__name__}: {e}"}
        out[key]["wall_s"] = round(time.time() - t0, 1)
        log(f"secondary {key}: {out[key]}")
        torch.cuda.empty_cache()
    return out


# ----------------------------------------------- 10M x 768 recall/QPS curves
def run_c5(args, cfg, name):
    """Per bit width: the plain search's recall@10/@100 and QPS against nprobe,
    and the learned search's against its confidence, with 100k queries in
    uneven batches through a plan (max_batch 4096).  Data, clustering (the
    library's k-means), index construction (the library's builder) and the
    ground truth on the GPU; nothing of that is timed."""
    import torch

    from erq_b200 import IVF, Plan, datasets, indexfile, learned, metrics
    from erq_b200.build_index import build_index_torch
    from erq_b200.clustering import kmeans

    torch.cuda.set_device(0)
    work = cache_dir(name, dict(cfg, bits=0))
    os.makedirs(work, exist_ok=True)
    t0 = time.time()
    nq_all = cfg["nq"] + cfg["qps_queries"] + cfg["train_queries"]
    base, qall = datasets.gaussian_mixture_torch(cfg["n"], cfg["dim"], cfg["comps"], cfg["sigma"],
                                                 cfg["seed"], nq_all, cfg["zipf"])
    log(f"c5: data at {time.time() - t0:.1f}s")
    cent, ids = kmeans(base, cfg["K"], iters=20, seed=cfg["seed"] + 1)
    log(f"c5: k-means at {time.time() - t0:.1f}s")
    q_eval = qall[:cfg["nq"]]
    q_qps = qall[cfg["nq"]:cfg["nq"] + cfg["qps_queries"]].cpu().numpy()
    q_train = qall[cfg["nq"] + cfg["qps_queries"]:].cpu().numpy()
    gt, _ = datasets.ground_truth_shortlist(base, q_eval, cfg["k"])
    gt = gt.cpu().numpy().astype(np.uint32)
    q_eval = q_eval.cpu().numpy()
    log(f"c5: ground truth at {time.time() - t0:.1f}s")
    rng = np.random.default_rng(cfg["seed"] + 5)
    sizes = []
    while sum(sizes) < cfg["qps_queries"]:
        sizes.append(int(min(cfg["max_batch"], np.exp(rng.uniform(0, np.log(cfg["max_batch"]))))))
    sizes[-1] -= sum(sizes) - cfg["qps_queries"]
    qd = torch.from_numpy(q_qps).cuda()
    k = cfg["k"]
    out = {}
    for bits in cfg["bits_list"]:
        path = os.path.join(work, f"ivf{bits}.index")
        tb = time.time()
        # the torch builder (plumbing): erq_build_index's exact fast_quantize
        # keeps a priority queue per vector in global memory and is meant for
        # reference-identical files, not for 10M vectors
        indexfile.write_index(path, build_index_torch(base, torch.from_numpy(cent).cuda(),
                                                      torch.from_numpy(ids.astype(np.int64)).cuda(),
                                                      bits, seed=cfg["seed"] + bits))
        build_s = time.time() - tb
        idx = IVF(path)
        res = {"build_s": round(build_s, 1), "plain": [], "learned": []}
        ids_d = torch.empty((cfg["max_batch"], k), dtype=torch.int32, device="cuda")

        def qps_of(plan, depth):
            """QPS over the uneven batch sequence; deep probes take a prefix
            of it (at least 8,192 queries) so one point stays under a minute."""
            st = torch.cuda.current_stream()
            budget = max(8192, int(cfg["qps_queries"] * min(1.0, 32.0 / max(depth, 1.0))))
            seq, tot = [], 0
            for b in sizes:
                if tot >= budget:
                    break
                seq.append(b)
                tot += b
            o = 0
            for b in seq[:8]:  # warm-up and graph capture of some sizes
                plan.search_buffers(qd[:b], ids_d[:b], stream=st)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for b in seq:
                plan.search_buffers(qd[o:o + b], ids_d[:b], stream=st)
                o += b
            e1.record(st)
            torch.cuda.synchronize()
            return tot / (e0.elapsed_time(e1) / 1e3), tot

        chosen = None
        prev = -1.0
        for nprobe in (1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024):
            if nprobe > cfg["K"]:
                break
            r_ids, _ = idx.search_raw(q_eval, k, nprobe, with_dists=False)
            r100 = metrics.recall_at_k(r_ids, gt, k)
            r10 = metrics.recall_at_k(r_ids[:, :10], gt[:, :10], 10)
            plan = Plan(idx, max_batch=cfg["max_batch"], k=k, nprobe=nprobe, raw=True)
            qps, nqps = qps_of(plan, nprobe)
            plan.free()
            res["plain"].append({"nprobe": nprobe, "recall@10": round(r10, 4),
                                 "recall@100": round(r100, 4), "qps": round(qps, 1),
                                 "qps_queries": nqps})
            log(f"c5 {bits}-bit nprobe {nprobe}: {res['plain'][-1]}")
            if chosen is None and r100 >= cfg["recall_target"]:
                chosen = nprobe
            # stop once recall saturates: the estimates' own error (the code
            # width) caps it below 1 at few bits
            if r100 > 0.995 or r100 - prev < 0.002:
                break
            prev = r100
        if chosen is not None:
            cfg_l = dict(cfg, bits=bits)
            model, meta = learned_model(idx, work, cfg_l, chosen, train=q_train)
            res["model"] = meta
            plan_l = Plan(idx, max_batch=cfg["max_batch"], k=k, nprobe=chosen, model=model, raw=True)
            for conf in (0.02, 0.1, 0.3, 0.5, 0.7, 0.9, 0.99):
                plan_l.set_learned(conf, LEARNED_MIN_PROB)
                ids_l, _, used = learned.search_learned(idx, model, idx.rotate(q_eval), k, chosen,
                                                        conf, LEARNED_MIN_PROB)
                qps, nqps = qps_of(plan_l, float(used.mean()))
                res["learned"].append({"confidence": conf, "mean_nprobe": round(float(used.mean()), 1),
                                       "recall@10": round(metrics.recall_at_k(ids_l[:, :10], gt[:, :10], 10), 4),
                                       "recall@100": round(metrics.recall_at_k(ids_l, gt, k), 4),
                                       "qps": round(qps, 1), "qps_queries": nqps})
                log(f"c5 {bits}-bit learned {res['learned'][-1]}")
            plan_l.free()
            model.free()
        res["plain_nprobe_at_target"] = chosen
        idx.free()
        out[f"{bits}-bit"] = res
        os.remove(path)
    print(json.dumps({"metric": "recall@10/100 and QPS curves, 10M x 768 Zipf, K=16384",
                      "workload": name, "data": cfg["data"], "batch_sizes": len(sizes),
                      "results": out}), flush=True)


# ---------------------------------------------------- batched latency mode
def run_latency(args, cfg, name):
    """Per batch size B of cfg["latency_batches"]: a plan autotuned for B,
    then calls of B queries (already in device memory) timed one by one with
    CUDA events; QPS = queries / summed call time, p50 / p99 of the calls."""
    import torch

    from erq_b200 import IVF, Plan, metrics

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if rank == 0:
        d = prepare(name, cfg)
    barrier(world)
    d = prepare(name, cfg) if rank != 0 else d
    index_path = os.path.join(d, "ivf.index")
    query = np.load(os.path.join(d, "query.npy"))
    gt = np.load(os.path.join(d, "gt.npy"))
    nq, k = query.shape[0], cfg["k"]
    idx = IVF(index_path, device=local)
    if args.nprobe:
        cfg = dict(cfg, nprobe=args.nprobe)
    nprobe, recall, ids0 = choose_nprobe(idx, query, gt, cfg)
    sizes = indexfile_sizes(index_path)
    stream = torch.cuda.current_stream()
    qd = torch.from_numpy(query).cuda()
    out = {}
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.mark_start()
    for B in cfg["latency_batches"]:
        plan = Plan(idx, max_batch=B, k=k, nprobe=nprobe, raw=True)
        tune, _ = plan.autotune(query[:B], reps=2)
        ids_d = torch.empty((B, k), dtype=torch.int32, device="cuda")
        calls = max(args.steps, min(2000, (4 * nq) // B))
        starts = list(range(0, nq - B + 1, B)) or [0]
        for w in range(args.warmup):
            s0 = starts[w % len(starts)]
            plan.search_buffers(qd[s0:s0 + B], ids_d, stream=stream)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(calls)]
        torch.cuda.synchronize()
        barrier(world)
        for c in range(calls):
            s0 = starts[c % len(starts)]
            ev[c][0].record(stream)
            plan.search_buffers(qd[s0:s0 + B], ids_d, stream=stream)
            ev[c][1].record(stream)
        torch.cuda.synchronize()
        lat = np.array([a.elapsed_time(b) for a, b in ev])
        tot = max_over_ranks(float(lat.sum()), world)
        # results equal the plain search's
        s0 = starts[(calls - 1) % len(starts)]
        assert (ids_d.cpu().numpy().view(np.uint32) == ids0[s0:s0 + B]).all()
        out[str(B)] = {"qps": round(world * B * calls / (tot / 1e3), 1),
                       "p50_ms": round(float(np.percentile(lat, 50)), 4),
                       "p99_ms": round(float(np.percentile(lat, 99)), 4),
                       "calls": calls, "tuning": tune}
        log(f"batch {B}: {out[str(B)]}")
        plan.free()
    clocks = sampler.stop() if sampler else None
    if rank == 0:
        big = str(max(cfg["latency_batches"]))
        print(json.dumps({
            "metric": f"QPS and per-batch p50/p99 latency, {name}", "value": out[big]["qps"],
            "unit": "queries/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": cfg["data"],
            "config": {"workload": f"{name}: batched plain plans, {cfg['n']}x{cfg['dim']}, "
                                   f"K={cfg['K']}, {cfg['bits']}-bit, top-{k}",
                       "nprobe": nprobe, "recall@100": round(recall, 5),
                       "cluster_sizes": {"min": int(sizes.min()), "median": int(np.median(sizes)),
                                         "max": int(sizes.max())}},
            "batches": out, "clocks": clocks}), flush=True)
    idx.free()
    dist_finish(world)


def indexfile_sizes(path):
    """Cluster sizes from the index header (N, DIM, K, EX, then K sizes)."""
    with open(path, "rb") as f:
        hdr = np.fromfile(f, np.uint64, 4)
        return np.fromfile(f, np.uint64, int(hdr[2])).astype(np.int64)


# ------------------------------------------------------------ reference arm
def run_reference(args, cfg, name):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    d = prepare(name, cfg)
    index_path = os.path.join(d, "ivf.index")
    query = np.load(os.path.join(d, "query.npy"))
    k, nq = cfg["k"], query.shape[0]
    searcher, kind, note = cpu_searcher(index_path)
    threads = os.cpu_count() or 1
    nprobe = cfg.get("nprobe")
    if not nprobe:
        # the recall-driven nprobe, found with the reference itself on a sample
        from erq_b200 import metrics

        gt = np.load(os.path.join(d, "gt.npy"))
        sub = min(500, nq)
        nprobe = NPROBE_SWEEP[-1]
        for p in NPROBE_SWEEP:
            if p > cfg["K"]:
                break
            if kind == "reference":
                qr = searcher.rotate(query[:sub])
                ids = searcher.search(qr, k, p, nthreads=threads)
            else:
                P = searcher.rotation()
                pad = np.zeros((sub, P.shape[0]), np.float32)
                pad[:, :query.shape[1]] = query[:sub]
                ids, _ = searcher.search(pad @ P, k, p, nthreads=threads)
            r = metrics.recall_at_k(ids, gt[:sub], k)
            log(f"reference nprobe={p}: recall@{k}={r:.4f} (first {sub} queries)")
            if r >= cfg["recall_target"]:
                nprobe = p
                break
    per_step = []
    samples = []
    offset = 0
    # each step a bounded sample, so that the whole run stays near two minutes
    step_s = min(args.ref_step_s, max(0.3, 120.0 / (args.warmup + args.steps)))
    for s in range(args.warmup + args.steps):
        qs = np.roll(query, -offset, axis=0)
        qps, n, sec, _, _ = time_cpu(searcher, kind, qs, k, nprobe, threads, step_s, nq)
        offset = (offset + n) % nq
        if s >= args.warmup:
            per_step.append(sec)
            samples.append(n)
    total_q, total_s = sum(samples), sum(per_step)
    value = total_q / total_s
    out = {
        "metric": METRIC, "impl": "reference", "value": round(value, 2), "unit": "queries/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * total_s / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": cfg["data"],
        "config": {"workload": f"{name}: the reference's IVF::search (AVX-512 CPU) on samples "
                               f"of the {nq}-query batch, top-{k}", "nprobe": nprobe},
        "cpu_baseline": {"value": round(value, 2), "unit": "queries/s", "cores": threads,
                         "kind": kind,
                         "sample": f"{args.steps} steps of ~{step_s:.2f}s each, "
                                   f"{total_q} queries total at nprobe={nprobe} incl. the "
                                   "reference's own query rotation" + (f"; {note}" if note else "")},
        "e2e": {"value": round(value, 2), "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    searcher.close()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default=DEFAULT_CONFIG)
    ap.add_argument("--cpu-budget", type=float, default=15.0,
                    help="seconds of CPU search for the cpu_baseline sample")
    ap.add_argument("--ref-step-s", type=float, default=6.0,
                    help="seconds of CPU search per step of the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer e2e timing")
    ap.add_argument("--no-learned", action="store_true", help="plain fixed-nprobe search only")
    ap.add_argument("--no-depth-sweep", action="store_true",
                    help="skip the plain-path scan timing at nprobe 16 and 64")
    ap.add_argument("--no-batched", action="store_true", help="skip the plain batched plan")
    ap.add_argument("--queries", type=int, default=0,
                    help="use only the first N queries of the batch (profiling cases)")
    ap.add_argument("--nprobe", type=int, default=0,
                    help="start the recall sweep at this nprobe")
    ap.add_argument("--prep-only", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the other workloads (small 128-d, 4-bit, Zipf learned) reported "
                         "under 'secondary' of the headline run")
    args = ap.parse_args()
    if args.warmup < 3 and not args.prep_only:
        log("warm-up raised to the minimum of 3 steps")
        args.warmup = 3
    cfg = CONFIGS[args.config]
    if args.prep_only:
        print(prepare(args.config, cfg))
        return
    if args.impl == "reference":
        run_reference(args, cfg, args.config)
    else:
        if cfg.get("c5"):
            run_c5(args, cfg, args.config)
        elif cfg.get("latency_batches"):
            run_latency(args, cfg, args.config)
        else:
            out = run_ours(args, cfg, args.config)
            if out is not None:
                if args.gpus == 1 and args.config == DEFAULT_CONFIG and not args.no_secondary:
                    out["secondary"] = run_secondary(args)
                print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
