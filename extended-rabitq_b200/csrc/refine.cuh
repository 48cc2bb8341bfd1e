// Lower-bound test, EX-bit refinement and the per-query top-k pool.
//
// One warp per query replays the reference's sequential scan order
// (inc/index/IVF.hpp:313-321, inc/index/HASearcher.hpp:82-112,187-236):
// clusters in probe order, blocks in storage order, candidates of a block in
// ascending lane order.  The block's candidate mask is taken against the
// top-k threshold as it stands when the block starts; every candidate is
// offered to the pool in order and the threshold is refreshed after each
// insertion.  The integer sums S come from the scan kernel; everything that
// depends on the threshold happens here, so the candidate sets and the
// returned ids and distances equal the reference's.
//
//   lower bound  accumulate_one_block_high_acc  inc/index/fastscan/FastScan.hpp:295-323
//   ex-IP        IP16_fxu8 / IP32_fxu4 / IP64_fxu{2,3,6,7}  inc/utils/space.hpp
//   distance     inc/index/HASearcher.hpp:225-232
//   pool         ResultPool::insert / distk    inc/index/Pool.hpp:15-31
#pragma once

#include <cfloat>

#include "common.cuh"

namespace erq {

struct RefineArgs {
    const float* qrot;            // [nq][D]
    const float* centroids;       // [K][D]
    const uint32_t* probe_cid;    // [nq][nprobe]
    const float* probe_sqy;       // [nq][nprobe]
    const uint64_t* s_off;        // [nq][nprobe]
    const int32_t* S;
    const float* qp_delta;        // [nq][nprobe]
    const float* qp_sumq;         // [nq][nprobe]
    const float* onorm;           // [blocks*32]
    const uint8_t* excode;        // [N][D*EX/8]
    const float* xipnorm;         // [N]
    const uint32_t* ids;          // [N]
    const uint32_t* c_first_block; // [K]
    const uint32_t* c_first_vec;   // [K]
    const uint32_t* c_size;        // [K]
    uint32_t* out_ids;            // [nq][k]
    float* out_dists;             // [nq][k] or null
    const int* q_nprobe;          // optional [nq]: clusters probed by each query
    int nq, D, EX, nprobe, k;
};


// float(v) for 0 <= v < 256 held in byte `i` of `w`: 0x4B0000vv is 2^23 + v.
__device__ __forceinline__ float byte_to_float(uint32_t w, int i) {
    return __fsub_rn(__int_as_float((int)__byte_perm(w, 0x4B000000u, 0x7540u | (uint32_t)i)),
                     8388608.f);
}

// Four consecutive dims (16*sub + 4*qd .. +3 of a 64-dim group) of one EX-bit
// code as bytes of a word.  `w` holds the group's 8*EX bytes as 2*EX words.
// Layouts: store_compacted_code, inc/index/Quantizer.hpp:491-631.
template <int EX>
__device__ __forceinline__ uint32_t ex_quad(const uint32_t* w, int sub, int qd) {
    if (EX == 8) {
        return w[4 * sub + qd];
    } else if (EX == 4) {  // per 32 dims: 16 bytes, low nibble = dims 0-15
        const uint32_t c = w[4 * (sub >> 1) + qd];
        return (sub & 1) ? ((c >> 4) & 0x0F0F0F0Fu) : (c & 0x0F0F0F0Fu);
    } else if (EX == 2 || EX == 3) {  // 2 bits at 2*sub of bytes 0-15
        uint32_t v = (w[qd] >> (2 * sub)) & 0x03030303u;
        if (EX == 3) {
            // bit j of byte m of the top word = bit 2 of dim 8j + m; these
            // dims have m = (4qd .. 4qd+3) % 8 and j = 2*sub + qd/2
            const uint32_t t = w[4 + (qd & 1)];
            const int j = 2 * sub + (qd >> 1);
            v |= ((j <= 2) ? (t << (2 - j)) : (t >> (j - 2))) & 0x04040404u;
        }
        return v;
    } else {  // EX == 6 || EX == 7: c1 = bytes 0-15, c2 = 16-31, c3 = 32-47
        const uint32_t c1 = w[qd], c2 = w[4 + qd], c3 = w[8 + qd];
        uint32_t v;
        if (sub == 0) {
            v = c1 & 0x3F3F3F3Fu;
        } else if (sub == 1) {
            v = c2 & 0x3F3F3F3Fu;
        } else if (sub == 2) {
            v = ((c1 >> 2) & 0x30303030u) | (c3 & 0x0F0F0F0Fu);
        } else {
            v = ((c2 >> 2) & 0x30303030u) | ((c3 >> 4) & 0x0F0F0F0Fu);
        }
        if (EX == 7) {  // bit 6 from the top word (after 48 bytes)
            const uint32_t t = w[12 + (qd & 1)];
            const int j = 2 * sub + (qd >> 1);
            v |= ((j <= 6) ? (t << (6 - j)) : (t >> (j - 6))) & 0x40404040u;
        }
        return v;
    }
}

// <unit_q, ex code> computed by one thread in the reference's order:
// accumulator l takes fma(unit_q[16s+l], code[16s+l], acc[l]) for s = 0,1,...
// then the reduce tree (IP*_fxu* in inc/utils/space.hpp).  unit_q is in
// shared memory and read as broadcasts (all lanes walk the same dims).
template <int EX>
__device__ __forceinline__ float ex_ip_thread(const float* __restrict__ uq,
                                              const uint8_t* __restrict__ code, int D) {
    float acc[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) acc[l] = 0.f;
    const uint2* src = reinterpret_cast<const uint2*>(code);
    for (int t = 0; t < (D >> 6); ++t) {
        uint32_t w[2 * EX];
#pragma unroll
        for (int i = 0; i < EX; ++i) {
            const uint2 x = __ldg(src + EX * t + i);
            w[2 * i] = x.x;
            w[2 * i + 1] = x.y;
        }
        const float4* u4 = reinterpret_cast<const float4*>(uq + 64 * t);
#pragma unroll
        for (int sub = 0; sub < 4; ++sub) {
#pragma unroll
            for (int qd = 0; qd < 4; ++qd) {
                const uint32_t v = ex_quad<EX>(w, sub, qd);
                const float4 u = u4[4 * sub + qd];
                acc[4 * qd + 0] = __fmaf_rn(u.x, byte_to_float(v, 0), acc[4 * qd + 0]);
                acc[4 * qd + 1] = __fmaf_rn(u.y, byte_to_float(v, 1), acc[4 * qd + 1]);
                acc[4 * qd + 2] = __fmaf_rn(u.z, byte_to_float(v, 2), acc[4 * qd + 2]);
                acc[4 * qd + 3] = __fmaf_rn(u.w, byte_to_float(v, 3), acc[4 * qd + 3]);
            }
        }
    }
    float t3[8], t6[4];
#pragma unroll
    for (int l = 0; l < 8; ++l) t3[l] = __fadd_rn(acc[l + 8], acc[l]);
#pragma unroll
    for (int m = 0; m < 4; ++m) t6[m] = __fadd_rn(t3[m + 4], t3[m]);
    return __fadd_rn(__fadd_rn(t6[0], t6[2]), __fadd_rn(t6[1], t6[3]));
}

constexpr int kRefineThreads = 128;     // 4 warps per query
constexpr int kWindowBlocks = 16;       // blocks whose candidates are refined together
constexpr int kWindowLanes = kWindowBlocks * 32;

// Shared memory of one block: unit_q[D] | per window lane: lb, ipq, onorm,
// ex_dist, id, list | pool_d[kpad] | pool_id[kpad] | misc
__host__ __device__ constexpr size_t refine_smem_bytes_per_query(int D, int kpad) {
    return (size_t)D * 4 + (size_t)kWindowLanes * (5 * 4 + 2) + (size_t)kpad * 8 + 64 + 128;
}

// Order key: ascending distance (-0 equal to +0, as float compares see it);
// among equal distances the higher lane, offered to the pool later, first.
// Non-candidates sort last.
__device__ __forceinline__ uint64_t merge_key(float d, int lane, bool cand) {
    const uint32_t b = __float_as_uint(d == 0.f ? 0.f : d);
    const uint32_t o = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return cand ? (((uint64_t)o << 32) | (uint32_t)(31 - lane)) : ~0ull;
}

// Offers one block's candidates (lanes with `cand`, distance d, id) to the
// pool in ascending lane order, as ResultPool::insert does one at a time
// (inc/index/Pool.hpp:15-26), in one parallel step.  Each insert keeps the k
// smallest entries under the order (distance, newer first): lower_bound
// places a new value before equal ones, an equal value still enters a full
// pool and pushes the last one out, a larger one is rejected.  A sequence of
// inserts therefore leaves the k smallest of (pool + sequence) in that order:
// sort the candidates by (distance, later lane first); pool entry i moves to
// i + #(candidates <= it), candidate j goes to j + #(pool entries < it), and
// ranks >= k fall off.  Executed by one whole warp; `cs` is 32 floats of
// scratch.
__device__ __forceinline__ void pool_merge_block(float* pool_d, uint32_t* pool_id, int& size, int k,
                                                 float& distk, bool cand, float d, uint32_t id,
                                                 float* cs, int lane) {
    const int nc = __popc(__ballot_sync(0xffffffffu, cand));
    uint64_t key = merge_key(d, lane, cand);
    uint32_t val = id;
    float dv = d;
#pragma unroll
    for (int sz = 2; sz <= 32; sz <<= 1) {
#pragma unroll
        for (int st = sz >> 1; st > 0; st >>= 1) {
            const uint64_t ok = __shfl_xor_sync(0xffffffffu, key, st);
            const uint32_t ov = __shfl_xor_sync(0xffffffffu, val, st);
            const float od = __shfl_xor_sync(0xffffffffu, dv, st);
            const bool take_min = ((lane & st) == 0) == ((lane & sz) == 0);
            if (take_min ? (ok < key) : (ok > key)) {
                key = ok;
                val = ov;
                dv = od;
            }
        }
    }
    // lane j holds the j-th candidate
    cs[lane] = dv;
    int lo = 0;
    if (lane < nc) {
        int hi = size;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (pool_d[mid] < dv) lo = mid + 1; else hi = mid;
        }
    }
    const int rc = lane < nc ? lane + lo : k;
    const int first = __shfl_sync(0xffffffffu, lo, 0);  // entries below it stay put
    __syncwarp();
    // move pool entries, top chunk first: entry i goes to i + c(i) >= i, and
    // i + c(i) strictly increases with i, so no chunk overwrites an entry
    // that has not been read or one already moved
    for (int i0 = ((size - 1) >> 5) << 5; i0 >= 0 && i0 + 31 >= first; i0 -= 32) {
        const int i = i0 + lane;
        float pd = 0.f;
        uint32_t pid = 0u;
        int pr = k;
        if (i < size) {
            pd = pool_d[i];
            pid = pool_id[i];
            int l2 = 0, h2 = nc;
            while (l2 < h2) {
                const int mid = (l2 + h2) >> 1;
                if (cs[mid] <= pd) l2 = mid + 1; else h2 = mid;
            }
            pr = i + l2;
        }
        __syncwarp();
        if (pr < k) {
            pool_d[pr] = pd;
            pool_id[pr] = pid;
        }
        __syncwarp();
    }
    if (rc < k) {
        pool_d[rc] = dv;
        pool_id[rc] = val;
    }
    __syncwarp();
    size = min(k, size + nc);
    distk = size == k ? pool_d[k - 1] : FLT_MAX;
}

// One block of 4 warps per query.  Per window of up to 16 blocks of the
// current cluster: every warp computes the lower bounds of 4 blocks and lists
// the lanes below the threshold as it stands at the window's start (a superset
// of the exact candidates, because the threshold only falls); all 128 threads
// refine the listed candidates, one each; warp 0 then replays the window in
// the reference's order - each block's mask against the threshold at that
// block's start, candidates in ascending lane order - inserting into the pool.
template <int EX>
__global__ void __launch_bounds__(kRefineThreads) refine_kernel(RefineArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = blockIdx.x;
    const int D = a.D, k = a.k;
    const int kpad = (k + 31) & ~31;
    float* uq = reinterpret_cast<float*>(smem_raw);
    float* w_lb = uq + D;
    float* w_ipq = w_lb + kWindowLanes;
    float* w_on = w_ipq + kWindowLanes;
    float* w_ed = w_on + kWindowLanes;
    uint32_t* w_id = reinterpret_cast<uint32_t*>(w_ed + kWindowLanes);
    uint16_t* w_list = reinterpret_cast<uint16_t*>(w_id + kWindowLanes);
    float* pool_d = reinterpret_cast<float*>(w_list + kWindowLanes);
    uint32_t* pool_id = reinterpret_cast<uint32_t*>(pool_d + kpad);
    int* misc = reinterpret_cast<int*>(pool_id + kpad);  // [0] list count [1] pool size
    float* s_distk = reinterpret_cast<float*>(misc + 2);
    float* cs = reinterpret_cast<float*>(misc + 16);  // 32 floats of merge scratch
    const int code_len = D * EX / 8;
    const int fac_rescale = 1 << EX;
    const float one_over_sqrtD = recip_via_double(__fsqrt_rn((float)D));
    const float* qv = a.qrot + (size_t)q * D;

    for (int i = tid; i < kpad; i += blockDim.x) {
        pool_d[i] = 0.f;
        pool_id[i] = 0u;
    }
    if (tid == 0) {
        *s_distk = FLT_MAX;
        misc[1] = 0;  // pool size as seen by all warps
    }
    int size = 0;         // pool state, maintained by warp 0
    float distk = FLT_MAX;
    __syncthreads();

    const int np_q = a.q_nprobe ? a.q_nprobe[q] : a.nprobe;
    for (int p = 0; p < np_q; ++p) {
        const size_t qp = (size_t)q * a.nprobe + p;
        const uint32_t cid = a.probe_cid[qp];
        const float sqy = a.probe_sqy[qp];
        const float y = __fsqrt_rn(sqy);
        const float delta = a.qp_delta[qp];
        const float sumq = a.qp_sumq[qp];
        // lower-bound constants (inc/index/fastscan/FastScan.hpp:297-303)
        const float c1 = __double2float_rn(__dsub_rn(__dmul_rn(0.5, (double)sumq), (double)kConstBound));
        const float c2 = __fmul_rn(__fmul_rn(-5.f, y), one_over_sqrtD);
        const float c3 = __fmul_rn(y, y);
        const double ex_sub = __dmul_rn((double)fac_rescale - 0.5, (double)sumq);
        const uint32_t n = a.c_size[cid];
        const uint32_t fb = a.c_first_block[cid];
        const uint32_t first_vec = a.c_first_vec[cid];
        const int32_t* S = a.S + a.s_off[qp];
        const uint32_t nblocks = (n + 31) >> 5;
        bool uq_ready = false;
        for (uint32_t wb = 0; wb < nblocks;) {
            const float d0 = *s_distk;
            const int filled = misc[1];
            // While the pool is filling every lane is a candidate: take just
            // enough blocks to fill it, so few lanes are refined in vain.
            const int want = filled < k ? min(kWindowBlocks, max(1, (k - filled + 31) / 32))
                                        : kWindowBlocks;
            const int nbw = (int)min((uint32_t)want, nblocks - wb);
            __syncthreads();
            if (tid == 0) misc[0] = 0;
            __syncthreads();
            // lower bounds and the candidate superset, 4 blocks per warp
#pragma unroll
            for (int i = 0; i < kWindowBlocks / (kRefineThreads / 32); ++i) {
                const int b = warp * (kWindowBlocks / (kRefineThreads / 32)) + i;
                if (b < nbw) {  // uniform per warp
                    const uint32_t blk = wb + b;
                    const float ipq = __fmul_rn(__int2float_rn(S[32 * blk + lane]), delta);
                    const float on = a.onorm[(size_t)(fb + blk) * 32 + lane];
                    float t = __fsub_rn(ipq, c1);
                    t = __fmul_rn(t, c2);
                    t = __fmul_rn(t, on);
                    t = __fadd_rn(t, c3);
                    t = __fadd_rn(t, __fmul_rn(on, on));
                    const bool valid = 32 * blk + lane < n;
                    // padding lanes never pass (NaN compares false)
                    w_lb[32 * b + lane] = valid ? t : __int_as_float(0x7fc00000);
                    w_ipq[32 * b + lane] = ipq;
                    w_on[32 * b + lane] = on;
                    const uint32_t m = __ballot_sync(0xffffffffu, valid && t < d0);
                    int base = 0;
                    if (lane == 0 && m) base = atomicAdd(&misc[0], __popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if ((m >> lane) & 1u)
                        w_list[base + __popc(m & ((1u << lane) - 1u))] = (uint16_t)(32 * b + lane);
                }
            }
            __syncthreads();
            const int cnt = misc[0];
            if (cnt == 0) {  // uniform: nothing in this window can pass
                wb += nbw;
                continue;
            }
            if (!uq_ready) {
                const float* cv = a.centroids + (size_t)cid * D;
                if (y > kNormEps) {
                    const float fac = recip_via_double(y);
                    for (int i = tid; i < D; i += blockDim.x) uq[i] = __fmul_rn(__fsub_rn(qv[i], cv[i]), fac);
                } else {
                    const float fill = recip_via_double(__fsqrt_rn((float)D));
                    for (int i = tid; i < D; i += blockDim.x) uq[i] = fill;
                }
                uq_ready = true;
                __syncthreads();
            }
            // refine the listed candidates, one per thread (idle threads repeat
            // the first so each warp stays converged on the broadcast reads)
            for (int r = 0; r < cnt; r += blockDim.x) {
                const int i = r + tid;
                const int slot = w_list[i < cnt ? i : 0];
                const size_t pos = (size_t)first_vec + 32 * wb + slot;
                const float ip = ex_ip_thread<EX>(uq, a.excode + pos * code_len, D);
                if (i < cnt) {
                    // inc/index/HASearcher.hpp:225-232
                    const float on = w_on[slot];
                    const float sqr_x = __fmul_rn(on, on);
                    const float t = __fadd_rn(__fmul_rn((float)fac_rescale, w_ipq[slot]), ip);
                    const double br = __dsub_rn((double)t, ex_sub);
                    const float xy = __fmul_rn(a.xipnorm[pos], y);
                    const float f = __fadd_rn(sqr_x, sqy);
                    w_ed[slot] = __double2float_rn(__dsub_rn((double)f, __dmul_rn((double)xy, br)));
                    w_id[slot] = a.ids[pos];
                }
            }
            __syncthreads();
            if (warp == 0) {
                for (int b = 0; b < nbw; ++b) {
                    const bool cand = w_lb[32 * b + lane] < distk;
                    if (__ballot_sync(0xffffffffu, cand))
                        pool_merge_block(pool_d, pool_id, size, k, distk, cand, w_ed[32 * b + lane],
                                         w_id[32 * b + lane], cs, lane);
                }
                if (lane == 0) {
                    *s_distk = distk;
                    misc[1] = size;
                }
            }
            __syncthreads();
            wb += nbw;
        }
    }
    if (warp == 0) {
        uint32_t* oid = a.out_ids + (size_t)q * k;
        for (int i = lane; i < k; i += 32) {
            oid[i] = i < size ? pool_id[i] : 0u;
            if (a.out_dists)
                a.out_dists[(size_t)q * k + i] = i < size ? pool_d[i] : __int_as_float(0x7f800000);
        }
    }
}

}  // namespace erq
