// Oracle harness over the reference's own search code (test infrastructure).
//
// Compiled against the unmodified reference headers (inc/) with the shim in
// oracle/shim standing in for Eigen and hnswlib.  Private members are opened
// with a macro so the per-stage state of the reference's HASearcher and
// ResultPool can be read; nothing in the reference is edited.  Exposes a
// plain C ABI for the Python tests (ctypes) and for the CPU baseline timing.
//
// Every entry point runs the reference's code: IVF::load, IVF::search,
// FlatInitializer::centroids_distances, HASearcher::preparing,
// accumulate_one_block_high_acc, the selected IP_FUNC and ResultPool.
// ref_trace/ref_search_dists step through IVF::search's own sequence
// (inc/index/IVF.hpp:295-324, inc/index/HASearcher.hpp:82-112,187-236) so that
// the candidate sequence and the pool's distances can be recorded; tests
// check that their ids equal IVF::search's.
#include <bits/stdc++.h>  // every standard header the reference pulls in, before the macro below
#include <immintrin.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#define HIGH_ACC_FAST_SCAN
#define EIGEN_DONT_PARALLELIZE
#define private public
#include "index/IVF.hpp"
#undef private

namespace {

struct RefIndex {
    IVF ivf;
};

// Silence the reference's progress prints during load.
struct CoutSilencer {
    std::streambuf* old;
    std::ofstream null;
    CoutSilencer() : old(std::cout.rdbuf()), null("/dev/null") { std::cout.rdbuf(null.rdbuf()); }
    ~CoutSilencer() { std::cout.rdbuf(old); }
};

// One step of HASearcher::scan_one_block (inc/index/HASearcher.hpp:187-236)
// with each refined candidate recorded before it is offered to the pool.
void traced_scan_one_block(HASearcher& s, uint8_t* block, float* block_fac, PID* ids,
                           float sqr_y, float y, float& distk, const Cluster& cur_cluster,
                           ResultPool& KNNs, size_t scanned_block, size_t num_points,
                           std::vector<std::pair<PID, float>>* trace) {
    const float* factor_x = s.DQ.factor_x2(block_fac);
    uint32_t mask = accumulate_one_block_high_acc(
        block, s.HC_LUT, factor_x, s.sumq, y, s.delta, s.shift, s.lower_distances,
        s.ip_xb_qprime, s.one_over_sqrtD, distk, s.D);
    // first num_points lanes (all 32 for a full block)
    mask = num_points >= 32 ? mask : (mask & ((1u << num_points) - 1));
    while (mask) {
        uint32_t lb = lowbit(mask);
        uint32_t j = bit_id(lb);
        mask -= lb;
        PID id = ids[j];
        float sqr_x = factor_x[j] * factor_x[j];
        size_t idx = j + scanned_block * FAST_SIZE;
        uint8_t* long_code = cur_cluster.long_code(idx, s.DQ);
        ExFactor ex_fac = *cur_cluster.ex_factor(idx);
        float ex_dist = sqr_x + sqr_y -
                        ex_fac.xipnorm * y *
                            (s.FAC_RESCALE * s.ip_xb_qprime[j] +
                             s.IP_FUNC(s.unit_q, long_code, s.D) - (s.FAC_RESCALE - 0.5) * s.sumq);
        if (trace) trace->emplace_back(id, ex_dist);
        KNNs.insert(id, ex_dist);
        distk = KNNs.distk();
    }
}

// IVF::search (inc/index/IVF.hpp:295-324) with tracing and pool access.
void traced_search(const IVF& ivf, const float* query, size_t k, size_t nprobe, PID* results,
                   float* dists, std::vector<std::pair<PID, float>>* trace) {
    std::vector<Candidate> centroid_dist(nprobe);
    ivf.initer->centroids_distances(query, nprobe, centroid_dist);
    ResultPool KNNs(k);
    HASearcher searcher(query, ivf.D, ivf.EX_BITS, ivf.DQ);
    for (size_t i = 0; i < nprobe; ++i) {
        PID cid = centroid_dist[i].id;
        float sqr_y = centroid_dist[i].distance;
        float* cur_centroid = ivf.initer->centroid(cid);
        const Cluster& cur_cluster = ivf.ClusterLst[cid];
        // HASearcher::search_cluster (inc/index/HASearcher.hpp:82-112)
        float y = std::sqrt(sqr_y);
        searcher.preparing(cur_centroid, y);
        size_t ITER = cur_cluster.iter();
        size_t REMAIN = cur_cluster.remain();
        uint8_t* block = cur_cluster.first_block();
        PID* ids = cur_cluster.ids();
        float distk = KNNs.distk();
        for (size_t b = 0; b < ITER; ++b) {
            float* block_fac = ivf.DQ.block_factor(block);
            traced_scan_one_block(searcher, block, block_fac, ids, sqr_y, y, distk, cur_cluster,
                                  KNNs, b, FAST_SIZE, trace);
            block = ivf.DQ.next_block(block_fac);
            ids = &ids[FAST_SIZE];
        }
        if (REMAIN > 0) {
            float* block_fac = ivf.DQ.block_factor(block);
            traced_scan_one_block(searcher, block, block_fac, ids, sqr_y, y, distk, cur_cluster,
                                  KNNs, ITER, REMAIN, trace);
        }
    }
    KNNs.copy_results(results);
    if (dists) {
        for (size_t i = 0; i < k; ++i)
            dists[i] = i < KNNs.size_ ? KNNs.distances_[i] : std::numeric_limits<float>::infinity();
    }
}

}  // namespace

extern "C" {

void* ref_load(const char* path) {
    std::ifstream probe(path, std::ios::binary);
    if (!probe.is_open()) return nullptr;
    probe.close();
    auto* r = new RefIndex();
    CoutSilencer quiet;
    r->ivf.load(path);
    return r;
}

void ref_free(void* h) { delete static_cast<RefIndex*>(h); }

void ref_info(void* h, uint64_t* out) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    out[0] = ivf.N;
    out[1] = ivf.DIM;
    out[2] = ivf.D;
    out[3] = ivf.K;
    out[4] = ivf.EX_BITS;
}

// IVF::search for each query, nthreads > 1 spreads queries over OpenMP
// threads (search is reentrant with the flat initializer).
void ref_search(void* h, const float* qrot, uint64_t nq, uint64_t k, uint64_t nprobe,
                uint32_t* ids, int nthreads) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    const size_t D = ivf.D;
    if (nthreads <= 1) {
        for (uint64_t q = 0; q < nq; ++q) ivf.search(qrot + q * D, nullptr, k, nprobe, ids + q * k);
        return;
    }
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int64_t q = 0; q < (int64_t)nq; ++q) ivf.search(qrot + q * D, nullptr, k, nprobe, ids + q * k);
}

// Same as ref_search, returns the wall time in seconds.
double ref_search_timed(void* h, const float* qrot, uint64_t nq, uint64_t k, uint64_t nprobe,
                        uint32_t* ids, int nthreads) {
    auto t0 = std::chrono::steady_clock::now();
    ref_search(h, qrot, nq, k, nprobe, ids, nthreads);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Step-through of IVF::search that also returns the pool's distances
// (unfilled slots: id 0 as in ResultPool::copy_results, distance +inf).
void ref_search_dists(void* h, const float* qrot, uint64_t nq, uint64_t k, uint64_t nprobe,
                      uint32_t* ids, float* dists) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    for (uint64_t q = 0; q < nq; ++q)
        traced_search(ivf, qrot + q * ivf.D, k, nprobe, ids + q * k, dists + q * k, nullptr);
}

// Every refined candidate (id, ex_dist) in the order the reference offers it
// to the pool.  Returns the total count (entries beyond cap are dropped).
uint64_t ref_trace(void* h, const float* qrot, uint64_t k, uint64_t nprobe, uint64_t cap,
                   uint32_t* cand_ids, float* cand_dist) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    std::vector<std::pair<PID, float>> trace;
    std::vector<PID> res(k);
    traced_search(ivf, qrot, k, nprobe, res.data(), nullptr, &trace);
    for (size_t i = 0; i < trace.size() && i < cap; ++i) {
        cand_ids[i] = trace[i].first;
        cand_dist[i] = trace[i].second;
    }
    return trace.size();
}

// FlatInitializer::centroids_distances: nprobe nearest centroids ascending.
void ref_probe(void* h, const float* qrot, uint64_t nprobe, uint32_t* cids, float* sqr_y) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    std::vector<Candidate> cd(nprobe);
    ivf.initer->centroids_distances(qrot, nprobe, cd);
    for (size_t i = 0; i < nprobe; ++i) {
        cids[i] = cd[i].id;
        sqr_y[i] = cd[i].distance;
    }
}

// All K centroid distances by the reference's L2Sqr16 (inc/utils/space.hpp:18-39).
void ref_centroid_dists(void* h, const float* qrot, float* out) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    for (size_t c = 0; c < ivf.K; ++c) out[c] = L2Sqr16(qrot, ivf.initer->centroid(c), ivf.D);
}

// HASearcher::preparing for one (query, cluster): unit_q[D], quantised query
// qq[D], delta, sumq, shift and the packed byte LUT (8*D bytes).
void ref_prepare(void* h, const float* qrot, uint32_t cid, float sqr_y, float* unit_q,
                 int16_t* qq, float* delta, float* sumq, int32_t* shift, uint8_t* lut) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    HASearcher s(qrot, ivf.D, ivf.EX_BITS, ivf.DQ);
    float y = std::sqrt(sqr_y);
    s.preparing(ivf.initer->centroid(cid), y);
    std::memcpy(unit_q, s.unit_q, sizeof(float) * ivf.D);
    std::memcpy(qq, s.quant_query, sizeof(int16_t) * ivf.D);
    *delta = s.delta;
    *sumq = s.sumq;
    *shift = s.shift;
    std::memcpy(lut, s.HC_LUT, s.TABLE_LENGTH * 2);
}

// accumulate_one_block_high_acc over every block of one cluster at a fixed
// distk: ipq[32*nblocks] and the raw lower-bound masks (before the
// remainder-lane cut).  Returns the number of blocks.
uint64_t ref_scan_cluster(void* h, const float* qrot, uint32_t cid, float sqr_y, float distk,
                          float* ipq, uint32_t* masks) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    HASearcher s(qrot, ivf.D, ivf.EX_BITS, ivf.DQ);
    float y = std::sqrt(sqr_y);
    s.preparing(ivf.initer->centroid(cid), y);
    const Cluster& cl = ivf.ClusterLst[cid];
    size_t nblocks = cl.iter() + (cl.remain() > 0);
    uint8_t* block = cl.first_block();
    for (size_t b = 0; b < nblocks; ++b) {
        float* block_fac = ivf.DQ.block_factor(block);
        masks[b] = accumulate_one_block_high_acc(block, s.HC_LUT, ivf.DQ.factor_x2(block_fac), s.sumq,
                                                 y, s.delta, s.shift, s.lower_distances,
                                                 s.ip_xb_qprime, s.one_over_sqrtD, distk, ivf.D);
        std::memcpy(ipq + 32 * b, s.ip_xb_qprime, sizeof(float) * 32);
        block = ivf.DQ.next_block(block_fac);
    }
    return nblocks;
}

// The EX-bit code inner product IP_FUNC(unit_q, long_code) for the vector at
// position `pos` of the index's long-code array (cluster order).
float ref_ex_ip(void* h, const float* unit_q, uint64_t pos) {
    const IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    HASearcher s(unit_q, ivf.D, ivf.EX_BITS, ivf.DQ);
    // IP_FUNC reads unit_q with aligned loads; copy into the searcher's buffer.
    std::memcpy(s.unit_q, unit_q, sizeof(float) * ivf.D);
    return s.IP_FUNC(s.unit_q, ivf.LONG_CODE + pos * ivf.DQ.long_code_length(), ivf.D);
}

// Rotator::rotate (inc/index/Rotator.hpp:60-63) of nq queries padded DIM->D.
void ref_rotate(void* h, const float* q, uint64_t nq, float* qrot) {
    IVF& ivf = static_cast<RefIndex*>(h)->ivf;
    FloatRowMat padded(nq, ivf.D);
    padded.setZero();
    for (uint64_t i = 0; i < nq; ++i) std::memcpy(&padded(i, 0), q + i * ivf.DIM, sizeof(float) * ivf.DIM);
    FloatRowMat rotated(nq, ivf.D);
    ivf.rotator().rotate(padded, rotated);
    std::memcpy(qrot, rotated.data(), sizeof(float) * nq * ivf.D);
}

float ref_l2sqr16(const float* x, const float* y, uint64_t L) { return L2Sqr16(x, y, L); }

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
