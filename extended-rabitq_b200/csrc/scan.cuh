// Per-(query, probed cluster) preparation and the FastScan accumulation.
//
// One thread block per (query q, probe rank p):
//   1. unit_q = (q_r - c) * (float)(1.0/y), max |unit_q|      normalize_query16,
//      data_range16               inc/utils/space.hpp:749-778, 608-628
//   2. delta = vmax / 8191, qq = round-half-away(unit_q / delta)
//                                 high_acc_quantize16, inc/utils/space.hpp:695-711
//   3. sumq = 16-lane ordered sum of unit_q (normalize_query16's return value)
//   4. 16-entry tables per 4-dim group: entry e = sum of qq[4g+b] over the bits
//      of e (bit 3 -> dim 4g+0)   pack_high_acc_LUT, inc/index/HASearcher.hpp:128-185
//   5. S_v = sum_g table_g[nibble_g(v)] = <x_b(v), qq> for every vector of
//      the cluster, exact int32     accumulate_one_block_high_acc,
//                                   inc/index/fastscan/FastScan.hpp:214-308
// S, delta and sumq go to global memory; the lower bound and the refinement
// that depend on the running top-k threshold happen in refine.cuh.
//
// Shared-memory tables: int16 entries, 16 per group (32 bytes).  For chunk c
// (groups 16c..16c+15) the tables occupy 512 bytes = two 256-byte windows;
// group 16c + 8h + u lives in window c*2 + u/4 at offset (u%4)*64 + h*32.
// At lookup step u the two half-warps (h = 0, 1) read different 8-bank sets,
// and the 16 lanes of a half-warp read one table: conflict-free.  The byte
// offset inside a window is formed from the code byte with a shift, a mask
// and a constant (2*nibble + 64u + 32h), and merged with the 256-aligned
// window address by one byte permute.
#pragma once

#include "common.cuh"

namespace erq {

struct ScanArgs {
    const float* qrot;        // [nq][D] rotated queries
    const float* centroids;   // [K][D] rotated centroids
    const uint32_t* probe_cid; // [nq][nprobe]
    const float* probe_sqy;   // [nq][nprobe]
    const uint8_t* codes;     // device block layout (layout.cuh)
    const uint32_t* c_first_block; // [K]
    const uint32_t* c_nblocks;     // [K]
    const uint64_t* s_off;    // [nq][nprobe] int32 offsets into S
    int32_t* S;               // output sums
    float* qp_delta;          // [nq][nprobe]
    float* qp_sumq;           // [nq][nprobe]
    const int* q_nprobe;      // optional [nq]: probe only the first q_nprobe[q] clusters
    const uint32_t* order;    // optional: block i scans pair order[i]
    const float* onorm;       // [blocks*32] (for the block minima)
    const uint32_t* c_size;   // [K]
    float* bmin;              // optional: smallest lower bound of each scanned block,
                              // at s_off/32 + block
    int D;
    int nprobe;
};

constexpr int kScanWarps = 4;

__device__ __forceinline__ int lds_s16(uint32_t addr) {
    int v;
    asm volatile("ld.shared.s16 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}
__device__ __forceinline__ int lds_s16_w1(uint32_t addr) {
    int v;
    asm volatile("ld.shared.s16 %0, [%1+256];" : "=r"(v) : "r"(addr));
    return v;
}

// 8 lookups for one 32-bit word of codes (4 groups u0..u0+3, one byte
// position).  `lo2`/`hi2` already hold 2*nibble + 64u + 32h per byte.
template <bool kWindow1>
__device__ __forceinline__ void lookup4(uint32_t lo2, uint32_t hi2, uint32_t base,
                                        int& acc_lo, int& acc_hi) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const uint32_t a = __byte_perm(lo2, base, 0x7650u | u);
        const uint32_t b = __byte_perm(hi2, base, 0x7650u | u);
        if (kWindow1) {
            acc_lo += lds_s16_w1(a);
            acc_hi += lds_s16_w1(b);
        } else {
            acc_lo += lds_s16(a);
            acc_hi += lds_s16(b);
        }
    }
}

__global__ void __launch_bounds__(kScanWarps * 32) scan_kernel(ScanArgs a) {
    extern __shared__ uint8_t smem_raw[];
    const int D = a.D;
    const int nchunk = D >> 6;
    const int ngroup = D >> 2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // carve shared memory: [pad to 256][tables nchunk*512][unit_q D floats][red]
    const uint32_t raw_s = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = (256u - (raw_s & 255u)) & 255u;
    uint8_t* tables = smem_raw + pad;
    const uint32_t tables_s = raw_s + pad;
    float* unit_q = reinterpret_cast<float*>(tables + nchunk * 512);
    float* red = unit_q + D;

    const uint32_t pair = a.order ? a.order[blockIdx.x] : blockIdx.x;
    const uint32_t q = pair / (uint32_t)a.nprobe;
    if (a.q_nprobe && (int)(pair - q * (uint32_t)a.nprobe) >= a.q_nprobe[q]) return;
    const uint32_t cid = a.probe_cid[pair];
    const float sqy = a.probe_sqy[pair];
    const float y = __fsqrt_rn(sqy);
    const bool normal = y > kNormEps;
    const float fac = normal ? recip_via_double(y) : 0.f;
    const float fill = recip_via_double(__fsqrt_rn((float)D));
    const float4* qv = reinterpret_cast<const float4*>(a.qrot + (size_t)q * D);
    const float4* cv = reinterpret_cast<const float4*>(a.centroids + (size_t)cid * D);

    // 1. unit_q and max |unit_q|
    float vmax = 0.f;
    for (int g = tid; g < ngroup; g += blockDim.x) {
        float4 u;
        if (normal) {
            const float4 x = qv[g], c = cv[g];
            u.x = __fmul_rn(__fsub_rn(x.x, c.x), fac);
            u.y = __fmul_rn(__fsub_rn(x.y, c.y), fac);
            u.z = __fmul_rn(__fsub_rn(x.z, c.z), fac);
            u.w = __fmul_rn(__fsub_rn(x.w, c.w), fac);
        } else {
            u = make_float4(fill, fill, fill, fill);
        }
        reinterpret_cast<float4*>(unit_q)[g] = u;
        vmax = fmaxf(vmax, fmaxf(fmaxf(fabsf(u.x), fabsf(u.y)), fmaxf(fabsf(u.z), fabsf(u.w))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if (lane == 0) red[warp] = vmax;
    __syncthreads();
    vmax = red[0];
#pragma unroll
    for (int w = 1; w < kScanWarps; ++w) vmax = fmaxf(vmax, red[w]);
    const float delta = __fdiv_rn(vmax, 8191.f);

    // 3. sumq on warp 0 (16 ordered chains + tree), written once
    if (warp == 0) {
        float acc = 0.f;
        if (lane < 16)
            for (int i = lane; i < D; i += 16) acc = __fadd_rn(acc, unit_q[i]);
        const float s = tree16_sum(acc);
        if (lane == 0) {
            const float sq = normal ? s : __fmul_rn((float)D, fill);
            a.qp_sumq[pair] = sq;
            a.qp_delta[pair] = delta;
            red[kScanWarps + 1] = sq;  // for the block minima, read after the barrier below
        }
    }

    // 2 + 4. quantise and build the group tables
    for (int g = tid; g < ngroup; g += blockDim.x) {
        const float4 u = reinterpret_cast<const float4*>(unit_q)[g];
        const int x0 = quantize_round(__fdiv_rn(u.x, delta));
        const int x1 = quantize_round(__fdiv_rn(u.y, delta));
        const int x2 = quantize_round(__fdiv_rn(u.z, delta));
        const int x3 = quantize_round(__fdiv_rn(u.w, delta));
        uint32_t packed[8];
#pragma unroll
        for (int e = 0; e < 16; e += 2) {
            const int v0 = ((e & 8) ? x0 : 0) + ((e & 4) ? x1 : 0) + ((e & 2) ? x2 : 0);
            const int v1 = v0 + x3;  // entry e+1 differs only in bit 0 (dim 4g+3)
            packed[e >> 1] = ((uint32_t)v0 & 0xffffu) | ((uint32_t)v1 << 16);
        }
        const int c = g >> 4, w = g & 15, h = w >> 3, u8 = w & 7;
        uint4* dst = reinterpret_cast<uint4*>(tables + c * 512 + (u8 >> 2) * 256 + (u8 & 3) * 64 +
                                              h * 32);
        dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
        dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
    }
    if (tid == 0) reinterpret_cast<uint32_t*>(red)[kScanWarps] = tables_s;
    __syncthreads();
    // The lookups below are inline PTX; their addresses derive from this
    // shared-memory read, which cannot move above the barrier.
    const uint32_t tables_base = reinterpret_cast<volatile uint32_t*>(red)[kScanWarps];

    // 5. scan: warp w takes blocks w, w + kScanWarps, ...
    const uint32_t nb = a.c_nblocks[cid];
    const uint8_t* cl_codes = a.codes + (size_t)a.c_first_block[cid] * (4 * D);
    int32_t* out = a.S + a.s_off[pair];
    const uint32_t h = lane >> 4, j = lane & 15;
    const uint32_t kconst = 0xC0804000u | (h ? 0x20202020u : 0u);
    // vector of this lane's output: perm0[j] for h = 0, perm0[j] + 16 for h = 1
    const uint32_t vout = ((j & 1) ? (j >> 1) + 8 : (j >> 1)) + 16 * h;
    const LbConsts lbk = lb_consts(red[kScanWarps + 1], y, recip_via_double(__fsqrt_rn((float)D)));
    const uint32_t csize = a.c_size[cid];
    const uint32_t fblock = a.c_first_block[cid];
    for (uint32_t b = warp; b < nb; b += kScanWarps) {
        const uint2* src = reinterpret_cast<const uint2*>(cl_codes + (size_t)b * (4 * D)) + lane;
        int acc_lo = 0, acc_hi = 0;
#pragma unroll 4
        for (int c = 0; c < nchunk; ++c) {
            const uint2 w = __ldg(src + c * 32);
            const uint32_t base = tables_base + c * 512;
            const uint32_t lo0 = ((w.x << 1) & 0x1E1E1E1Eu) | kconst;
            const uint32_t hi0 = ((w.x >> 3) & 0x1E1E1E1Eu) | kconst;
            lookup4<false>(lo0, hi0, base, acc_lo, acc_hi);
            const uint32_t lo1 = ((w.y << 1) & 0x1E1E1E1Eu) | kconst;
            const uint32_t hi1 = ((w.y >> 3) & 0x1E1E1E1Eu) | kconst;
            lookup4<true>(lo1, hi1, base, acc_lo, acc_hi);
        }
        // combine the two half-warps (even / odd group halves)
        acc_lo += __shfl_xor_sync(0xffffffffu, acc_lo, 16);
        acc_hi += __shfl_xor_sync(0xffffffffu, acc_hi, 16);
        const int sv = h ? acc_hi : acc_lo;
        out[32 * b + vout] = sv;
        if (a.bmin) {
            const float on = a.onorm[(size_t)(fblock + b) * 32 + vout];
            const float lb = lower_bound(__fmul_rn(__int2float_rn(sv), delta), on, lbk);
            const float m = warp_min(32 * b + vout < csize ? lb : INFINITY);
            if (lane == 0) a.bmin[a.s_off[pair] / 32 + b] = m;
        }
    }
}

}  // namespace erq
