// Coarse probe from tensor-core distance estimates, exact by construction.
//
// FlatInitializer::centroids_distances (inc/index/Initializer.hpp:55-68)
// ranks all K centroids by L2Sqr16 (inc/utils/space.hpp:18-39) and keeps the
// nprobe nearest.  Here the GEMM of gemm.cuh gives an estimate a_c of every
// squared distance with |a_c - true_c| <= eps_a, and one thread block per query
//   1. selects the Msel smallest estimates (radix select on order-preserving
//      keys) and sorts them by estimate; A = the (Msel+1)-th smallest estimate
//      bounds every centroid outside the list;
//   2. recomputes the exact reference value e_c (16 ordered FMA chains + the
//      reduce tree) of the first n = nprobe of the list, e_max = their largest;
//   3. finds the first list position P >= n whose estimate satisfies
//      a_P - eps > e_max, eps = eps_a + the reference's own rounding bound.
//      Every centroid at or after P (and outside the list) then has
//      e_c >= a_c - eps > e_max >= the n-th smallest exact distance, so the
//      exact top n lie in the first P: those are recomputed and sorted by
//      (e_c, c);
//   4. when no list position qualifies, all Msel are recomputed and the cut is
//      checked as A - eps > e_(n); if that fails too, probe_fallback_kernel
//      computes e_c for all K centroids and sorts them all.
// Usually P is a few positions past n, so few centroid rows are read.
#pragma once

#include "common.cuh"

namespace erq {

struct ProbeArgs {
    const float* approx;      // [nq][K] distance estimates
    const float* qrot;        // [nq][D]
    const float* centroids;   // [K][D] in chain order (chain_pos)
    const float* qn;          // [nq] squared query norms
    const uint32_t* c_nblocks; // [K]
    float cn_max;             // largest squared centroid norm
    float eps_rel;            // eps = eps_rel * (qn + cn_max)
    uint64_t stride;          // scan workspace per query (int32 entries)
    uint32_t* probe_cid;      // [nq][nprobe]
    float* probe_sqy;         // [nq][nprobe]
    uint64_t* s_off;          // [nq][nprobe]
    uint32_t* fallbacks;      // optional counter of queries that took step 4
    float* near_d;            // optional [nq][64]: the 64 smallest distance estimates, ascending
    int nq, K, Kpow2, D, nprobe, M;
    int Spow2;                // sort-key capacity of probe_kernel (probe_smem_bytes)
    uint32_t* fallback_flag;  // [nq]: 1 when the query needs probe_fallback_kernel
    int check_rank;           // rank whose exactness the bound check proves (>= nprobe)
    int stage_keys;           // nonzero: probe_kernel copies the K order keys to shared
                              // memory once (K <= kProbeStageKeys)
    uint64_t* sort_global;    // optional [nq][sort_cap]: sort keys in global memory, for
                              // selections too large for shared memory
    uint64_t sort_cap;        // keys per query in sort_global
    float* exact_rows;        // [nq][K]: probe_exact_kernel's exact distances (it may
                              // overwrite the estimates there)
    // probe_warp_kernel in two launches (<1>, then <2>; <0>: one launch):
    // <1> selects, sorts and writes the features, and keeps each query's
    // sorted list here; <2> finishes from it with the per-query check rank
    // q_check (the depth a probe model chose in between)
    uint64_t* list;           // [nq][kProbeWarpCap]
    uint32_t* list_n;         // [nq]
    uint64_t* list_cut;       // [nq]
    const int* q_check;       // [nq] (phase 2)
};

constexpr int kProbeThreads = 256;
constexpr int kProbeFeatRank = 64;  // estimates written to near_d
constexpr int kProbeStageKeys = 4096;  // largest K whose keys are staged in shared memory
constexpr int kProbeSortSmemKeys = 16384;  // largest sort kept in shared memory (128 KB)

__device__ __forceinline__ uint32_t order_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float order_key_value(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Probe copy of the centroids in accumulator-chain order: L2Sqr16's
// accumulator l (0..15) takes dims l, l+16, l+32, ... in turn; position
// (s * 16 + l) * 4 + i holds dim l + 16 * (4s + i).  Lane l of a half-warp then
// reads its accumulator's next four dims as one float4 at step s, the 16
// lanes 256 contiguous bytes.  D is a multiple of 64.
__host__ __device__ __forceinline__ int chain_pos(int d) {
    const int l = d & 15, j = d >> 4;
    return ((j >> 2) * 16 + l) * 4 + (j & 3);
}

__global__ void chain_layout_kernel(const float* __restrict__ in, int rows, int D,
                                    float* __restrict__ out) {
    const size_t n = (size_t)rows * D;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / D;
        const int d = (int)(i - r * D);
        out[r * D + chain_pos(d)] = in[i];
    }
}

// Exact L2Sqr16 of (q, centroid c) by the 16 lanes l of a half-warp, both in
// chain order: accumulator l takes t = q - c and fma(t, t, acc) over its dims
// in ascending order, then the reduce tree; valid in the half-warp's lane 0.
__device__ __forceinline__ float l2sqr16_chain(const float4* __restrict__ q4,
                                               const float4* __restrict__ c4, int D, int l) {
    float acc = 0.f;
#pragma unroll 2
    for (int s = 0; s < (D >> 6); ++s) {
        const float4 c = __ldg(c4 + s * 16 + l);
        const float4 x = q4[s * 16 + l];
        float t = __fsub_rn(x.x, c.x);
        acc = __fmaf_rn(t, t, acc);
        t = __fsub_rn(x.y, c.y);
        acc = __fmaf_rn(t, t, acc);
        t = __fsub_rn(x.z, c.z);
        acc = __fmaf_rn(t, t, acc);
        t = __fsub_rn(x.w, c.w);
        acc = __fmaf_rn(t, t, acc);
    }
    return tree16_sum(acc);
}

// Bitonic sort of n (power of two) 64-bit keys in shared memory, ascending.
__device__ __forceinline__ void block_bitonic_sort(uint64_t* keys, int n) {
    for (int size = 2; size <= n; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < (n >> 1); t += blockDim.x) {
                const int lo = 2 * t - (t & (stride - 1));
                const int hi = lo + stride;
                const bool up = (lo & size) == 0;
                const uint64_t a = keys[lo], b = keys[hi];
                if ((a > b) == up) {
                    keys[lo] = b;
                    keys[hi] = a;
                }
            }
            __syncthreads();
        }
    }
}

// Ascending sort of keys[0..n), n <= 64, by warp 0's lanes (element i in
// lane i % 32, register i / 32), bitonic network over 32 or 64 elements with
// the missing ones as ~0; no block barrier.
__device__ __forceinline__ void warp_sort64(uint64_t* keys, int n, int lane) {
    const int N = n <= 32 ? 32 : 64;
    uint64_t a = lane < n ? keys[lane] : ~0ull;
    uint64_t b = lane + 32 < n ? keys[lane + 32] : ~0ull;
    for (int size = 2; size <= N; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride == 32) {  // size 64: the pair sits in one lane
                const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
                a = lo;
                b = hi;
            } else {
                const bool low = (lane & stride) == 0;
                const uint64_t pa = __shfl_xor_sync(0xffffffffu, a, stride);
                const bool upa = (lane & size) == 0;
                a = (low == upa) ? (a < pa ? a : pa) : (a < pa ? pa : a);
                if (N == 64) {
                    const uint64_t pb = __shfl_xor_sync(0xffffffffu, b, stride);
                    const bool upb = ((lane + 32) & size) == 0;
                    b = (low == upb) ? (b < pb ? b : pb) : (b < pb ? pb : b);
                }
            }
        }
    }
    if (lane < n) keys[lane] = a;
    if (lane + 32 < n) keys[lane + 32] = b;
}

// Ascending sort of keys[0..n) by the whole block (called by every thread,
// after the keys are visible to all; returns synchronised).  Up to 64 keys
// warp 0 sorts them in registers; more are padded with ~0 to a power of two
// (keys must hold that many) and sorted by the block.
__device__ __forceinline__ void sort_prefix(uint64_t* keys, int n) {
    if (n <= 64) {
        if (threadIdx.x < 32) warp_sort64(keys, n, threadIdx.x);
        __syncthreads();
        return;
    }
    int np = 1;
    while (np < n) np <<= 1;
    for (int i = n + threadIdx.x; i < np; i += blockDim.x) keys[i] = ~0ull;
    __syncthreads();
    block_bitonic_sort(keys, np);
}

// Shared memory of probe_kernel: q[D] | order keys u32 [Kst] | sort keys u64
// [Spow2] | hist[256] | misc.  Kst = K rounded up to even when the keys are
// staged (stage_keys), else 0 and each radix pass re-reads the estimates
// from global memory.  Spow2 is a power of two >= the number of selected
// candidates (max(M, 64) with features, else M; K when all are selected);
// above kProbeSortSmemKeys the sort keys live in sort_global instead (pass
// Spow2 = 0 here).
__host__ __device__ constexpr size_t probe_smem_bytes(int D, int Spow2, int Kst) {
    return (size_t)D * 4 + (size_t)((Kst + 1) & ~1) * 4 + (size_t)Spow2 * 8 + 256 * 4 + 64;
}
// probe_exact_kernel: q[D] | hist[256] | misc | sort keys u64 [Npow2] (0 when
// they live in sort_global)
__host__ __device__ constexpr size_t probe_exact_smem_bytes(int D, int Npow2) {
    return (size_t)D * 4 + 256 * 4 + 64 + (size_t)Npow2 * 8;
}

// Radix select (8 bits per pass) of the rank-th smallest of the K order keys
// key_of(0..K-1), rank in 1..K; by the whole block, returns synchronised.
template <typename KeyOf>
__device__ uint32_t radix_select_key(KeyOf key_of, int K, int rank, uint32_t* hist, int* misc) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t prefix = 0, pmask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int c = tid; c < K; c += blockDim.x) {
            const uint32_t kk = key_of(c);
            if ((kk & pmask) == prefix) atomicAdd(&hist[(kk >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (warp == 0) {
            uint32_t h[8], s = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                h[i] = hist[8 * lane + i];
                s += h[i];
            }
            uint32_t incl = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const uint32_t excl = incl - s;
            if (excl < (uint32_t)rank && incl >= (uint32_t)rank) {
                uint32_t run = excl;
                int d = 0;
                for (; d < 8; ++d) {
                    if (run + h[d] >= (uint32_t)rank) break;
                    run += h[d];
                }
                misc[0] = 8 * lane + d;
                misc[1] = (int)run;
            }
        }
        __syncthreads();
        prefix |= (uint32_t)misc[0] << shift;
        pmask |= 0xffu << shift;
        rank -= misc[1];
        __syncthreads();
    }
    return prefix;
}

// Outputs of one query from its sorted (distance, id) keys, and the exclusive
// prefix of 32 * nblocks over the probe order; warp 0.
__device__ __forceinline__ void probe_outputs(const ProbeArgs& a, int q, const uint64_t* sorted,
                                              int lane) {
    uint64_t run = (uint64_t)q * a.stride;
    for (int p0 = 0; p0 < a.nprobe; p0 += 32) {
        const int p = p0 + lane;
        uint32_t nbv = 0;
        if (p < a.nprobe) {
            const uint64_t key = sorted[p];
            const uint32_t cid = (uint32_t)(key & 0xffffffffu);
            a.probe_cid[(size_t)q * a.nprobe + p] = cid;
            a.probe_sqy[(size_t)q * a.nprobe + p] = __uint_as_float((uint32_t)(key >> 32));
            nbv = 32u * a.c_nblocks[cid];
        }
        uint32_t incl = nbv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t n = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += n;
        }
        if (p < a.nprobe) a.s_off[(size_t)q * a.nprobe + p] = run + (incl - nbv);
        run += __shfl_sync(0xffffffffu, incl, 31);
    }
}

__global__ void __launch_bounds__(kProbeThreads) probe_kernel(ProbeArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int q = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int K = a.K, D = a.D;
    float* qs = reinterpret_cast<float*>(smem_raw);
    uint32_t* ks = reinterpret_cast<uint32_t*>(qs + D);
    const int Kst = a.stage_keys ? (K + 1) & ~1 : 0;
    uint64_t* sk_s = reinterpret_cast<uint64_t*>(ks + Kst);
    uint32_t* hist = reinterpret_cast<uint32_t*>(sk_s + (a.sort_global ? 0 : a.Spow2));
    int* misc = reinterpret_cast<int*>(hist + 256);  // [0] digit [1] before [2] count [3] ok
    uint64_t* sk = a.sort_global ? a.sort_global + (size_t)q * a.sort_cap : sk_s;

    for (int i = tid; i < D; i += blockDim.x) qs[chain_pos(i)] = a.qrot[(size_t)q * D + i];
    const float* aq = a.approx + (size_t)q * K;
    if (a.stage_keys)
        for (int c = tid; c < K; c += blockDim.x) ks[c] = order_key(__ldg(aq + c));
    // order key of centroid c's estimate (the staged copy is read only after
    // the barrier that follows the histogram reset)
    auto key_of = [&](int c) -> uint32_t { return a.stage_keys ? ks[c] : order_key(__ldg(aq + c)); };

    const int M = a.M;
    // with features requested the 64 smallest estimates are selected as well
    const int Msel = a.near_d ? max(M, kProbeFeatRank) : M;
    const bool select_all = Msel + 1 > K;
    uint32_t kstar = 0xffffffffu;
    if (!select_all) kstar = radix_select_key(key_of, K, Msel + 1, hist, misc);
    // candidates: every centroid whose estimate is below the (Msel+1)-th,
    // keyed by (estimate, id)
    if (tid == 0) misc[2] = 0;
    __syncthreads();
    for (int c = tid; c < K; c += blockDim.x) {
        const uint32_t kk = key_of(c);
        if (select_all || kk < kstar) {
            const int slot = atomicAdd(&misc[2], 1);
            sk[slot] = ((uint64_t)kk << 32) | (uint64_t)c;
        }
    }
    __syncthreads();
    const int ns = misc[2];
    const bool truncated = !select_all;  // A = value of kstar bounds the rest
    sort_prefix(sk, ns);
    if (a.near_d) {
        // the 64 smallest estimates, in order, are the distance features;
        // ranks the list misses are ties at the cut, the (Msel+1)-th estimate
        const float fill = truncated ? order_key_value(kstar)
                                     : ns > 0 ? order_key_value((uint32_t)(sk[ns - 1] >> 32)) : 0.f;
        for (int j = tid; j < kProbeFeatRank; j += blockDim.x)
            a.near_d[(size_t)q * kProbeFeatRank + j] =
                j < ns ? order_key_value((uint32_t)(sk[j] >> 32)) : fill;
    }
    const int n = min(a.check_rank, ns);
    const float eps = a.eps_rel * (a.qn[q] + a.cn_max);
    if (tid == 0) {
        misc[4] = 0;   // largest exact distance of the first n (float bits)
        misc[5] = ns;  // P
    }
    __syncthreads();
    // exact distances of list positions [lo, hi), one half-warp each; a warp
    // with no position in a pass skips it, a half-warp past the end repeats
    // its neighbour (both halves take part in the reduce's shuffles)
    const int hw = tid >> 4, l = tid & 15, nhw = blockDim.x >> 4;
    auto exact_range = [&](int lo, int hi, bool track_max) {
        for (int base = lo; base < hi; base += nhw) {
            const int i0 = base + 2 * warp;
            if (i0 >= hi) continue;  // uniform per warp
            const int i = base + hw;
            const uint32_t c = (uint32_t)(sk[i < hi ? i : i0] & 0xffffffffu);
            const float e = l2sqr16_chain(reinterpret_cast<const float4*>(qs), reinterpret_cast<const float4*>(a.centroids + (size_t)c * D), D, l);
            if (l == 0 && i < hi) {
                sk[i] = dist_key(e, c);
                if (track_max) atomicMax(reinterpret_cast<unsigned*>(&misc[4]), __float_as_uint(e));
            }
        }
    };
    exact_range(0, n, true);
    __syncthreads();
    const float e_max = __uint_as_float((uint32_t)misc[4]);
    for (int i = n + tid; i < ns; i += blockDim.x)
        if (order_key_value((uint32_t)(sk[i] >> 32)) - eps > e_max) atomicMin(&misc[5], i);
    __syncthreads();
    const int P = misc[5];
    const bool proven = P < ns || !truncated || (order_key_value(kstar) - eps > e_max);
    exact_range(n, P, false);
    __syncthreads();
    sort_prefix(sk, P);
    // a query whose cut is not proven goes to probe_fallback_kernel
    if (tid == 0) {
        bool ok = ns >= a.check_rank;
        if (ok && !proven) {
            const float e_n = __uint_as_float((uint32_t)(sk[a.check_rank - 1] >> 32));
            const float A = order_key_value(kstar);
            ok = (A - eps > e_n) && (e_n == e_n);
        }
        a.fallback_flag[q] = ok ? 0u : 1u;
        misc[3] = ok ? 1 : 0;
        if (!ok && a.fallbacks) atomicAdd(a.fallbacks, 1u);
    }
    __syncthreads();
    if (misc[3] && warp == 0) probe_outputs(a, q, sk, lane);
}

// ---------------------------------------------------------------------------
// Warp-per-query form of probe_kernel for the common case (the Msel
// candidates fit kProbeWarpCap): the same four steps with the same results,
// each query on one warp of a block of kProbeWarpWarps, no block barrier.
// Step 1 reads the estimate row from global memory on every pass instead of
// staging it: one pass for the smallest and largest order key, then radix
// passes whose first digit is the 8 bits below the highest bit those two
// differ in (the bits above are common to every key), until the digit's
// bucket holding rank Msel + 1 ends at most kProbeWarpCap keys from the
// bottom - its end is then the cut A (every key outside the list is at or
// above it, and the list holds the Msel smallest) - or the last digit gives
// the (Msel + 1)-th key itself.  Steps 2-4 as probe_kernel, with a half-warp
// per exact distance.
constexpr int kProbeWarpWarps = 8;
constexpr int kProbeWarpCap = 128;  // list capacity: four sort keys per lane

// Shared memory of one warp: q[D] in chain order | hist[256] | list u64 [cap] | misc
__host__ __device__ constexpr size_t probe_warp_smem_per_warp(int D) {
    return (size_t)D * 4 + 256 * 4 + (size_t)kProbeWarpCap * 8 + 32;
}

// Ascending bitonic sort of 32 * R keys, element j * 32 + lane in v[j].
template <int R>
__device__ __forceinline__ void warp_sort_regs(uint64_t (&v)[R], int lane) {
    constexpr int N = 32 * R;
#pragma unroll
    for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= 32) {
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    const int pj = j ^ (stride >> 5);
                    if (pj > j) {
                        const bool up = ((j * 32 + lane) & size) == 0;
                        const uint64_t x = v[j], y = v[pj];
                        if ((x > y) == up) {
                            v[j] = y;
                            v[pj] = x;
                        }
                    }
                }
            } else {
                const bool low = (lane & stride) == 0;
#pragma unroll
                for (int j = 0; j < R; ++j) {
                    const uint64_t o = __shfl_xor_sync(0xffffffffu, v[j], stride);
                    const bool up = ((j * 32 + lane) & size) == 0;
                    v[j] = (low == up) ? (v[j] < o ? v[j] : o) : (v[j] < o ? o : v[j]);
                }
            }
        }
    }
}

// Ascending sort of keys[0..n), n <= kProbeWarpCap, by one warp.
__device__ __forceinline__ void warp_sort_list(uint64_t* keys, int n, int lane) {
    if (n <= 64) {
        warp_sort64(keys, n, lane);
        __syncwarp();
        return;
    }
    uint64_t v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = j * 32 + lane < n ? keys[j * 32 + lane] : ~0ull;
    warp_sort_regs<4>(v, lane);
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (j * 32 + lane < n) keys[j * 32 + lane] = v[j];
    __syncwarp();
}

// PHASE 0: the whole probe; 1: through the features, keeping the sorted list;
// 2: the rest from that list (ProbeArgs::phase documents the two launches).
template <int PHASE>
__global__ void __launch_bounds__(kProbeWarpWarps * 32) probe_warp_kernel(ProbeArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = blockIdx.x * kProbeWarpWarps + warp;
    if (q >= a.nq) return;  // whole warp; nothing below waits across warps
    const int K = a.K, D = a.D;
    uint8_t* base = smem_raw + (size_t)warp * probe_warp_smem_per_warp(D);
    float* qs = reinterpret_cast<float*>(base);
    uint32_t* hist = reinterpret_cast<uint32_t*>(qs + D);
    uint64_t* sk = reinterpret_cast<uint64_t*>(hist + 256);
    if (PHASE != 1)
        for (int i = lane; i < D; i += 32) qs[chain_pos(i)] = a.qrot[(size_t)q * D + i];
    const float* aq = a.approx + (size_t)q * K;
    const uint32_t lt = (1u << lane) - 1u;
    uint64_t kstar = 0;
    int ns = 0;
    if (PHASE == 2) {  // the list phase 1 kept
        ns = (int)a.list_n[q];
        kstar = a.list_cut[q];
        for (int j = lane; j < ns; j += 32) sk[j] = a.list[(size_t)q * kProbeWarpCap + j];
        __syncwarp();
    } else {
        // f(order key) for this lane's share of the row (128-bit loads when K % 4 == 0)
        auto each_key = [&](auto&& f) {
            if ((K & 3) == 0) {
                const float4* aq4 = reinterpret_cast<const float4*>(aq);
                for (int c4 = lane; c4 < (K >> 2); c4 += 32) {
                    const float4 v = __ldg(aq4 + c4);
                    f(order_key(v.x));
                    f(order_key(v.y));
                    f(order_key(v.z));
                    f(order_key(v.w));
                }
            } else {
                for (int c = lane; c < K; c += 32) f(order_key(__ldg(aq + c)));
            }
        };

        // 1. the smallest and largest order key
        uint32_t lo = 0xffffffffu, hi = 0u;
        each_key([&](uint32_t kk) {
            lo = min(lo, kk);
            hi = max(hi, kk);
        });
        lo = __reduce_min_sync(0xffffffffu, lo);
        hi = __reduce_max_sync(0xffffffffu, hi);
        const int Msel = a.near_d ? max(a.M, kProbeFeatRank) : a.M;
        kstar = (uint64_t)lo;  // all keys equal: nothing lies below the (Msel+1)-th
        if (lo != hi) {
            const int hb = 31 - __clz((int)(lo ^ hi));
            int s = max(hb - 7, 0), w = hb - s + 1;  // the digit: bits [s, s + w)
            uint64_t prefix = (uint64_t)lo >> (s + w) << (s + w);
            uint32_t below = 0;  // keys under the current range
            int rank = Msel + 1;
            for (;;) {
                for (int i = lane; i < 256; i += 32) hist[i] = 0;
                __syncwarp();
                const uint32_t dmask = (1u << w) - 1u;
                const uint64_t want = prefix >> (s + w);
                each_key([&](uint32_t kk) {
                    if (((uint64_t)kk >> (s + w)) == want) atomicAdd(&hist[(kk >> s) & dmask], 1u);
                });
                __syncwarp();
                uint32_t h[8], sum = 0;
    #pragma unroll
                for (int i = 0; i < 8; ++i) {
                    h[i] = hist[8 * lane + i];
                    sum += h[i];
                }
                uint32_t incl = sum;
    #pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const uint32_t excl = incl - sum;
                const bool mine = excl < (uint32_t)rank && incl >= (uint32_t)rank;
                // in the lane that holds it: the bin of rank, the keys below it, its count
                int d = 7;
                uint32_t run = excl, hdv = 0, acc = excl;
                bool found = false;
    #pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (!found && acc + h[i] >= (uint32_t)rank) {
                        found = true;
                        d = i;
                        run = acc;
                        hdv = h[i];
                    }
                    acc += h[i];
                }
                const int src = __ffs(__ballot_sync(0xffffffffu, mine)) - 1;
                const int dg = __shfl_sync(0xffffffffu, 8 * lane + d, src);
                const uint32_t before = __shfl_sync(0xffffffffu, run, src);
                const uint32_t hd = __shfl_sync(0xffffffffu, hdv, src);
                const uint64_t b_lo = prefix | ((uint64_t)dg << s);
                if (s == 0) {  // the (Msel+1)-th key itself
                    kstar = b_lo;
                    break;
                }
                if (below + before + hd <= (uint32_t)kProbeWarpCap) {  // the bucket's end
                    kstar = b_lo + (1ull << s);
                    break;
                }
                below += before;
                rank -= (int)before;
                prefix = b_lo;
                const int s2 = max(s - 8, 0);
                w = s - s2;
                s = s2;
            }
        }
        // the list: every centroid whose key is below kstar, keyed by (estimate, id)
        for (int c0 = 0; c0 < K; c0 += 32) {
            const int c = c0 + lane;
            const uint32_t kk = c < K ? order_key(__ldg(aq + c)) : 0xffffffffu;
            const bool in = c < K && (uint64_t)kk < kstar;
            const uint32_t m = __ballot_sync(0xffffffffu, in);
            if (in) sk[ns + __popc(m & lt)] = ((uint64_t)kk << 32) | (uint64_t)c;
            ns += __popc(m);
        }
        __syncwarp();
        warp_sort_list(sk, ns, lane);
        if (a.near_d) {
            // the 64 smallest estimates, in order, are the distance features;
            // ranks the list misses are ties at the cut, the (Msel+1)-th estimate
            // (a list cut at a bucket's end holds more than 64)
            const float fill = order_key_value((uint32_t)kstar);
            for (int j = lane; j < kProbeFeatRank; j += 32)
                a.near_d[(size_t)q * kProbeFeatRank + j] =
                    j < ns ? order_key_value((uint32_t)(sk[j] >> 32)) : fill;
        }
        if (PHASE == 1) {  // keep the list for phase 2
            for (int j = lane; j < ns; j += 32) a.list[(size_t)q * kProbeWarpCap + j] = sk[j];
            if (lane == 0) {
                a.list_n[q] = (uint32_t)ns;
                a.list_cut[q] = kstar;
            }
            return;
        }
    }
    // 2-3. exact distances of list positions [lo, hi), a half-warp each
    const int check = PHASE == 2 ? a.q_check[q] : a.check_rank;
    const int n = min(check, ns);
    const float eps = a.eps_rel * (a.qn[q] + a.cn_max);
    const int hw = lane >> 4, l = lane & 15;
    uint32_t e_max_bits = 0u;  // the largest of the first n, as unsigned float bits
    auto exact_range = [&](int p0, int p1) {
        for (int i0 = p0; i0 < p1; i0 += 2) {
            const int i = i0 + hw < p1 ? i0 + hw : i0;  // a half-warp past the end repeats
            const uint32_t c = (uint32_t)(sk[i] & 0xffffffffu);
            const float e = l2sqr16_chain(reinterpret_cast<const float4*>(qs),
                                          reinterpret_cast<const float4*>(a.centroids + (size_t)c * D), D, l);
            const float e0 = __shfl_sync(0xffffffffu, e, 0), e1 = __shfl_sync(0xffffffffu, e, 16);
            if (lane == 0) sk[i0] = dist_key(e0, (uint32_t)(sk[i0] & 0xffffffffu));
            if (lane == 16 && i0 + 1 < p1) sk[i0 + 1] = dist_key(e1, c);
            e_max_bits = max(e_max_bits, __float_as_uint(e0));
            if (i0 + 1 < p1) e_max_bits = max(e_max_bits, __float_as_uint(e1));
            __syncwarp();
        }
    };
    __syncwarp();
    exact_range(0, n);
    const float e_max = __uint_as_float(e_max_bits);
    int P = ns;
    for (int i0 = n; i0 < ns; i0 += 32) {
        const int i = i0 + lane;
        const bool qual = i < ns && order_key_value((uint32_t)(sk[i] >> 32)) - eps > e_max;
        const uint32_t m = __ballot_sync(0xffffffffu, qual);
        if (m) {
            P = i0 + __ffs(m) - 1;
            break;
        }
    }
    const bool truncated = kstar < (1ull << 32);
    const bool proven = P < ns || !truncated || (order_key_value((uint32_t)kstar) - eps > e_max);
    exact_range(n, P);
    warp_sort_list(sk, P, lane);
    // a query whose cut is not proven goes to probe_exact_kernel (so does one
    // whose list is shorter than the nprobe slots the outputs fill)
    bool ok = ns >= check && ns >= a.nprobe;
    if (ok && !proven) {
        const float e_n = __uint_as_float((uint32_t)(sk[check - 1] >> 32));
        const float A = order_key_value((uint32_t)kstar);
        ok = (A - eps > e_n) && (e_n == e_n);
    }
    if (lane == 0) {
        a.fallback_flag[q] = ok ? 0u : 1u;
        if (!ok && a.fallbacks) atomicAdd(a.fallbacks, 1u);
    }
    if (ok) probe_outputs(a, q, sk, lane);
}

// The exact nprobe nearest centroids of a query, by (distance, id), from all
// K exact distances - for the queries whose cut probe_kernel could not prove
// (fallback_flag set; `compute`: the exact L2Sqr16 values are computed here
// into the query's row of exact_rows, over its estimates), and for the
// allocation-free search, whose rows already hold them (fallback_flag null,
// compute 0).  A radix select finds the nprobe-th smallest key; the keys below
// it and, among those equal to it, the smallest ids fill nprobe slots, which
// are sorted (FlatInitializer::centroids_distances' partial_sort,
// inc/index/Initializer.hpp:55-68, with ties by id).  Sort keys live in
// shared memory up to kProbeSortSmemKeys, else in sort_global.
__global__ void __launch_bounds__(kProbeThreads) probe_exact_kernel(ProbeArgs a, int compute, int Npow2) {
    const int q = blockIdx.x;
    if (a.fallback_flag && !a.fallback_flag[q]) return;
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int K = a.K, D = a.D, n = min(a.nprobe, K);
    float* qs = reinterpret_cast<float*>(smem_raw);
    uint32_t* hist = reinterpret_cast<uint32_t*>(qs + D);
    int* misc = reinterpret_cast<int*>(hist + 256);
    uint64_t* sk = a.sort_global ? a.sort_global + (size_t)q * a.sort_cap
                                 : reinterpret_cast<uint64_t*>(misc + 16);
    float* row = a.exact_rows + (size_t)q * K;
    if (compute) {
        for (int i = tid; i < D; i += blockDim.x) qs[chain_pos(i)] = a.qrot[(size_t)q * D + i];
        __syncthreads();
        const int hw = tid >> 4, l = tid & 15, nhw = blockDim.x >> 4;
        for (int base = 0; base < K; base += nhw) {
            const int c = base + hw;
            const float e = l2sqr16_chain(reinterpret_cast<const float4*>(qs),
                                          reinterpret_cast<const float4*>(a.centroids + (size_t)min(c, K - 1) * D), D, l);
            if (l == 0 && c < K) row[c] = e;
        }
        __syncthreads();
    }
    auto key_of = [&](int c) -> uint32_t { return order_key(row[c]); };
    const uint32_t kstar = radix_select_key(key_of, K, n, hist, misc);
    if (tid == 0) misc[2] = 0;
    __syncthreads();
    for (int c = tid; c < K; c += blockDim.x) {
        const uint32_t kk = key_of(c);
        if (kk < kstar) sk[atomicAdd(&misc[2], 1)] = dist_key(order_key_value(kk), (uint32_t)c);
    }
    __syncthreads();
    if (warp == 0) {  // ties at the cut: the smallest ids, in ascending order
        int have = misc[2];
        for (int base = 0; base < K && have < n; base += 32) {
            const int c = base + lane;
            const bool eq = c < K && key_of(c) == kstar;
            const uint32_t m = __ballot_sync(0xffffffffu, eq);
            const int r = __popc(m & ((1u << lane) - 1u));
            if (eq && have + r < n) sk[have + r] = dist_key(order_key_value(kstar), (uint32_t)c);
            have += __popc(m);
        }
    }
    __syncthreads();
    for (int i = n + tid; i < Npow2; i += blockDim.x) sk[i] = ~0ull;
    __syncthreads();
    if (Npow2 <= 64) {
        if (warp == 0) warp_sort64(sk, n, lane);
        __syncthreads();
    } else {
        block_bitonic_sort(sk, Npow2);
    }
    if (warp == 0) probe_outputs(a, q, sk, lane);
}

}  // namespace erq
