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
    int nq, D, EX, nprobe, k;
};

constexpr int kRefineWarps = 4;

// Value of dim 16*s + l of one EX-bit code (store_compacted_code layouts,
// inc/index/Quantizer.hpp:491-631).
template <int EX>
__device__ __forceinline__ uint32_t ex_value(const uint8_t* __restrict__ code, int s, int l) {
    if (EX == 8) {
        return code[16 * s + l];
    } else if (EX == 4) {
        return (code[16 * (s >> 1) + l] >> (4 * (s & 1))) & 15u;
    } else if (EX == 2 || EX == 3) {
        constexpr int seg = (EX == 2) ? 16 : 24;
        const uint8_t* c = code + seg * (s >> 2);
        const int sub = s & 3;
        uint32_t v = (c[l] >> (2 * sub)) & 3u;
        if (EX == 3) {
            const int d = 16 * sub + l;  // dim within the 64-dim group
            const uint8_t tb = c[16 + (d & 7)];  // byte m = d % 8 of the top-bit word
            v |= ((tb >> (d >> 3)) & 1u) << 2;
        }
        return v;
    } else {  // EX == 6 || EX == 7
        constexpr int seg = (EX == 6) ? 48 : 56;
        const uint8_t* c = code + seg * (s >> 2);
        const int sub = s & 3;
        uint32_t v;
        if (sub == 0) {
            v = c[l] & 63u;
        } else if (sub == 1) {
            v = c[16 + l] & 63u;
        } else if (sub == 2) {
            v = ((uint32_t)(c[l] >> 6) << 4) | (c[32 + l] & 15u);
        } else {
            v = ((uint32_t)(c[16 + l] >> 6) << 4) | (c[32 + l] >> 4);
        }
        if (EX == 7) {
            const int d = 16 * sub + l;
            const uint8_t tb = c[48 + (d & 7)];
            v |= ((tb >> (d >> 3)) & 1u) << 6;
        }
        return v;
    }
}

// <unit_q, ex code>: lane l of the 16-lane segment accumulates
// fma(unit_q[16s+l], code[16s+l], acc) in ascending s; result in lane 0.
template <int EX>
__device__ __forceinline__ float ex_ip(const float* __restrict__ unit_q,
                                       const uint8_t* __restrict__ code, int D, int l) {
    float acc = 0.f;
    const int nsteps = D >> 4;
#pragma unroll 8
    for (int s = 0; s < nsteps; ++s)
        acc = __fmaf_rn(unit_q[16 * s + l], (float)ex_value<EX>(code, s, l), acc);
    return tree16_sum(acc);
}

template <int EX>
__global__ void __launch_bounds__(kRefineWarps * 32) refine_kernel(RefineArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = blockIdx.x * kRefineWarps + warp;
    if (q >= a.nq) return;
    const int D = a.D, k = a.k;
    const int kpad = (k + 31) & ~31;
    float* unit_q = reinterpret_cast<float*>(smem_raw) +
                    (size_t)warp * (D + 2 * kpad);
    float* pool_d = unit_q + D;
    uint32_t* pool_id = reinterpret_cast<uint32_t*>(pool_d + kpad);
    const int code_len = D * EX / 8;
    const int fac_rescale = 1 << EX;
    const float one_over_sqrtD = recip_via_double(__fsqrt_rn((float)D));
    const float* qv = a.qrot + (size_t)q * D;

    for (int i = lane; i < kpad; i += 32) {
        pool_d[i] = 0.f;
        pool_id[i] = 0u;
    }
    __syncwarp();
    int size = 0;
    float distk = FLT_MAX;

    for (int p = 0; p < a.nprobe; ++p) {
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
        for (uint32_t b = 0; b < nblocks; ++b) {
            const float ipq = __fmul_rn(__int2float_rn(S[32 * b + lane]), delta);
            const float on = a.onorm[(size_t)(fb + b) * 32 + lane];
            float lb = __fsub_rn(ipq, c1);
            lb = __fmul_rn(lb, c2);
            lb = __fmul_rn(lb, on);
            lb = __fadd_rn(lb, c3);
            lb = __fadd_rn(lb, __fmul_rn(on, on));
            const bool valid = 32 * b + lane < n;
            uint32_t mask = __ballot_sync(0xffffffffu, valid && (lb < distk));
            if (mask && !uq_ready) {
                // unit_q for the refinement (same arithmetic as the scan kernel)
                const float* cv = a.centroids + (size_t)cid * D;
                if (y > kNormEps) {
                    const float fac = recip_via_double(y);
                    for (int i = lane; i < D; i += 32)
                        unit_q[i] = __fmul_rn(__fsub_rn(qv[i], cv[i]), fac);
                } else {
                    const float fill = recip_via_double(__fsqrt_rn((float)D));
                    for (int i = lane; i < D; i += 32) unit_q[i] = fill;
                }
                __syncwarp();
                uq_ready = true;
            }
            while (mask) {
                // two candidates at a time, one per half-warp
                const int j0 = __ffs(mask) - 1;
                mask &= mask - 1;
                const int j1 = mask ? __ffs(mask) - 1 : -1;
                if (j1 >= 0) mask &= mask - 1;
                const int hw = lane >> 4, l = lane & 15;
                const int jm = hw ? (j1 >= 0 ? j1 : j0) : j0;
                const size_t pos = (size_t)first_vec + 32 * b + jm;
                const float ip = ex_ip<EX>(unit_q, a.excode + pos * code_len, D, l);
                // distance estimate in lane 0 of each half (HASearcher.hpp:225-232)
                const float ipq_j = __shfl_sync(0xffffffffu, ipq, jm);
                const float on_j = __shfl_sync(0xffffffffu, on, jm);
                float ex_dist = 0.f;
                uint32_t id = 0;
                if (l == 0) {
                    const float sqr_x = __fmul_rn(on_j, on_j);
                    const float t = __fadd_rn(__fmul_rn((float)fac_rescale, ipq_j), ip);
                    const double br = __dsub_rn((double)t, ex_sub);
                    const float xy = __fmul_rn(a.xipnorm[pos], y);
                    const float f = __fadd_rn(sqr_x, sqy);
                    ex_dist = __double2float_rn(__dsub_rn((double)f, __dmul_rn((double)xy, br)));
                    id = a.ids[pos];
                }
                const int ncand = j1 >= 0 ? 2 : 1;
                for (int t = 0; t < ncand; ++t) {
                    const float dnew = __shfl_sync(0xffffffffu, ex_dist, 16 * t);
                    const uint32_t inew = __shfl_sync(0xffffffffu, id, 16 * t);
                    // ResultPool::insert
                    if (size == k && dnew > pool_d[size - 1]) continue;
                    // lower_bound: number of entries < dnew
                    int lo = 0;
                    for (int i0 = 0; i0 < size; i0 += 32) {
                        const int i = i0 + lane;
                        const bool lt = i < size && pool_d[i] < dnew;
                        lo += __popc(__ballot_sync(0xffffffffu, lt));
                    }
                    // shift [lo, last) up by one; when full the entry at k-1
                    // falls off.  Chunks of 32 from the top down: each chunk is
                    // read before the chunk below writes into its first slot.
                    const int last = size < k ? size : k - 1;
                    for (int i0 = lo + ((last - lo - 1) >> 5) * 32; last > lo && i0 >= lo; i0 -= 32) {
                        const int i = i0 + lane;
                        float sv = 0.f;
                        uint32_t si = 0u;
                        if (i < last) {
                            sv = pool_d[i];
                            si = pool_id[i];
                        }
                        __syncwarp();
                        if (i < last) {
                            pool_d[i + 1] = sv;
                            pool_id[i + 1] = si;
                        }
                        __syncwarp();
                    }
                    if (lane == 0) {
                        pool_d[lo] = dnew;
                        pool_id[lo] = inew;
                    }
                    __syncwarp();
                    size += size < k;
                    distk = size == k ? pool_d[k - 1] : FLT_MAX;
                }
            }
        }
    }
    uint32_t* oid = a.out_ids + (size_t)q * k;
    for (int i = lane; i < k; i += 32) {
        oid[i] = i < size ? pool_id[i] : 0u;
        if (a.out_dists) a.out_dists[(size_t)q * k + i] = i < size ? pool_d[i] : __int_as_float(0x7f800000);
    }
}

}  // namespace erq
