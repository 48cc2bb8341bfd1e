// Work order for L2 reuse.  Many queries probe the same (often large)
// clusters; when the thread blocks that read one cluster run close together
// in time, its codes come from L2 instead of HBM for all but the first.  The
// order is a counting sort of work items by cluster id: (query, probe) pairs
// for the scan kernel, queries by their nearest cluster for the refinement
// kernel.  The order changes which block handles which item, never what an
// item computes.
#pragma once

#include "common.cuh"

namespace erq {

// key of (query, probe) pair i: its cluster, or K for pairs a per-query probe
// count leaves out (those blocks exit at once; they go last).
// With size_rank the key is the cluster's rank by decreasing size instead
// (one scan block per pair: the longest scans start first).
__global__ void pair_keys_kernel(const uint32_t* __restrict__ probe_cid, uint32_t pairs, int nprobe,
                                 const int* __restrict__ q_nprobe, uint32_t K,
                                 const uint32_t* __restrict__ size_rank,
                                 uint32_t* __restrict__ keys) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pairs) return;
    const uint32_t q = i / (uint32_t)nprobe, p = i - q * (uint32_t)nprobe;
    const uint32_t c = probe_cid[i];
    keys[i] = (q_nprobe && (int)p >= q_nprobe[q]) ? K : (size_rank ? size_rank[c] : c);
}

// key of query q: the rank, by decreasing size, of the cluster it probes
// first.  Queries of one cluster stay together (L2 reuse) and the queries
// with the most refinement work start first, so none of them is left for the
// last wave of thread blocks.
__global__ void query_keys_kernel(const uint32_t* __restrict__ probe_cid, uint32_t nq, int nprobe,
                                  const uint32_t* __restrict__ size_rank, uint32_t* __restrict__ keys) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nq) keys[q] = size_rank[probe_cid[(size_t)q * nprobe]];
}

// Lanes of a warp with equal keys add once (popular clusters and the
// left-out bucket would otherwise serialise on one counter).
__global__ void bucket_count_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                    uint32_t* __restrict__ counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    const uint32_t key = in ? keys[i] : 0xffffffffu;
    const uint32_t act = __ballot_sync(0xffffffffu, in);
    if (!in) return;
    const uint32_t peers = __match_any_sync(act, key);
    if ((threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&counts[key], (uint32_t)__popc(peers));
}

// In-place exclusive prefix sum of counts[nb], one block of 1024 threads.
constexpr int kBucketScanThreads = 1024;
__global__ void __launch_bounds__(kBucketScanThreads) bucket_scan_kernel(uint32_t* __restrict__ counts,
                                                                         uint32_t nb) {
    __shared__ uint32_t part[kBucketScanThreads];
    const uint32_t per = (nb + kBucketScanThreads - 1) / kBucketScanThreads;
    const uint32_t lo = min(nb, threadIdx.x * per), hi = min(nb, lo + per);
    uint32_t s = 0;
    for (uint32_t i = lo; i < hi; ++i) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < kBucketScanThreads; o <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - s;
    for (uint32_t i = lo; i < hi; ++i) {
        const uint32_t c = counts[i];
        counts[i] = run;
        run += c;
    }
}

__global__ void bucket_scatter_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                      uint32_t* __restrict__ offsets, uint32_t* __restrict__ order) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    const uint32_t key = in ? keys[i] : 0xffffffffu;
    const uint32_t act = __ballot_sync(0xffffffffu, in);
    if (!in) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t peers = __match_any_sync(act, key);
    const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&offsets[key], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, (int)leader);
    order[base + __popc(peers & ((1u << lane) - 1u))] = i;
}

}  // namespace erq
