// Work order for L2 reuse.  Many queries probe the same (often large)
// clusters; when the thread blocks that read one cluster run close together
// in time, its codes come from L2 instead of HBM for all but the first.  The
// order is a counting sort of work items by cluster: (query, probe) pairs for
// the scan kernels, queries by their nearest cluster for the refinement
// kernel.  The order changes which block handles which item, never what an
// item computes.
#pragma once

#include "common.cuh"

namespace erq {

// Lanes of a warp with equal keys add once (popular clusters and the
// left-out bucket would otherwise serialise on one counter).
__device__ __forceinline__ void count_key(bool in, uint32_t key, uint32_t* __restrict__ counts) {
    const uint32_t act = __ballot_sync(0xffffffffu, in);
    if (!in) return;
    const uint32_t peers = __match_any_sync(act, key);
    if ((threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&counts[key], (uint32_t)__popc(peers));
}

// Both sorts' keys and bucket counts in one pass (pairs >= nq; the grid
// covers pairs).  Pair i = (q, p): its cluster id, or with pairs_by_size the
// cluster's rank by decreasing size (one scan block per pair: the longest
// scans start first); K for pairs a per-query probe count leaves out (those
// blocks exit at once; they go last).  Query q: the size rank of the cluster
// it probes first, so the queries of one cluster stay together (L2 reuse) and
// those with the most refinement work start first.  Keys go to keys_p /
// keys_q, counts to counts_p / counts_q.
__global__ void order_keys_count_kernel(const uint32_t* __restrict__ probe_cid, uint32_t pairs,
                                        uint32_t nq, int nprobe, const int* __restrict__ q_nprobe,
                                        uint32_t K, bool pairs_by_size,
                                        const uint32_t* __restrict__ size_rank,
                                        uint32_t* __restrict__ keys_p, uint32_t* __restrict__ counts_p,
                                        uint32_t* __restrict__ keys_q, uint32_t* __restrict__ counts_q) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t kp = 0, kq = 0;
    if (i < pairs) {
        const uint32_t q = i / (uint32_t)nprobe, p = i - q * (uint32_t)nprobe;
        const uint32_t c = probe_cid[i];
        kp = (q_nprobe && (int)p >= q_nprobe[q]) ? K : (pairs_by_size ? size_rank[c] : c);
        keys_p[i] = kp;
    }
    if (i < nq) {
        kq = size_rank[probe_cid[(size_t)i * nprobe]];
        keys_q[i] = kq;
    }
    count_key(i < pairs, kp, counts_p);
    count_key(i < nq, kq, counts_q);
}

// In-place exclusive prefix sum of counts[nb], one block of 1024 threads.
constexpr int kBucketScanThreads = 1024;
// With a grid of two blocks, block 1 scans counts1.
__global__ void __launch_bounds__(kBucketScanThreads) bucket_scan_kernel(uint32_t* __restrict__ counts0,
                                                                         uint32_t* __restrict__ counts1,
                                                                         uint32_t nb) {
    __shared__ uint32_t part[kBucketScanThreads];
    uint32_t* counts = blockIdx.x == 0 ? counts0 : counts1;
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

__device__ __forceinline__ void scatter_key(const uint32_t* __restrict__ keys, uint32_t n,
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

// Both sorts' scatters (n0 >= n1; the grid covers n0).
__global__ void bucket_scatter2_kernel(const uint32_t* __restrict__ keys0, uint32_t n0,
                                       uint32_t* __restrict__ offsets0, uint32_t* __restrict__ order0,
                                       const uint32_t* __restrict__ keys1, uint32_t n1,
                                       uint32_t* __restrict__ offsets1, uint32_t* __restrict__ order1) {
    scatter_key(keys0, n0, offsets0, order0);
    scatter_key(keys1, n1, offsets1, order1);
}

}  // namespace erq
