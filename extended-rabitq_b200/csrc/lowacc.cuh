// The reference's second index format and searcher: built and searched when
// HIGH_ACC_FAST_SCAN is not defined (inc/index/Searcher.hpp,
// inc/index/Quantizer.hpp:33-37, 290-300).  Four factors per vector in each
// FastScan block (||o - c||^2, the inner-product factor, the number of set
// bits, the error factor), the query quantised to unsigned 14-bit values over
// [vl, vr] (Searcher::preparing, Searcher.hpp:121-126; minus_sum16,
// data_range16, scalar_quantize16 in inc/utils/space.hpp), and per block
//   rabitq_ip = (float)S * width + sumxb * vl - sum(q - c) / 2
//   lower     = (||o-c||^2 + y^2) - (rabitq_ip * fac_ip + fac_err * y)
// (Searcher::scan_one_block, Searcher.hpp:187-236); a vector is refined when
// lower <= the running k-th distance, tested lane by lane with the threshold
// refreshed after every insertion, and its distance is
//   ||o-c||^2 + y^2 - xipnorm * (2^EX * rabitq_ip + <q - c, ex code>
//                                - (2^EX - 1) * sum(q - c) / 2)      in float.
//
// S = sum_i x_i * qq_i is again an exact integer (the reference splits its
// 16-bit tables into bytes and sums them exactly, accumulate_robust,
// inc/index/fastscan/FastScan.hpp:139-212).  The scan here uses the 6-dim
// groups of scan.cuh with 32-bit table entries (a sum of six 14-bit values
// needs 17 bits): 64 entries = 256 bytes per group, code byte = 4 * idx, the
// group's table at + 256 i of its chunk (transform_blocks_kernel with
// entry_bytes = 4).
#pragma once

#include <cfloat>

#include "common.cuh"
#include "layout.cuh"
#include "refine.cuh"
#include "scan.cuh"

namespace erq {

__host__ __device__ constexpr uint32_t low_table_bytes(int D) { return (uint32_t)hex_chunks(D) * 4096u; }

template <int OFF>
__device__ __forceinline__ int lds_u32(uint32_t addr) {
    int v;
    asm("ld.shared.u32 %0, [%1+%2];" : "=r"(v) : "r"(addr), "n"(OFF));
    return v;
}

// 4 lookups of code word `word` (groups 4W .. 4W+3 of chunk base cb).
template <int W>
__device__ __forceinline__ int low_lookup4(uint32_t word, uint32_t cb) {
    const uint32_t a0 = __byte_perm(word, cb, 0x7650u), a1 = __byte_perm(word, cb, 0x7651u);
    const uint32_t a2 = __byte_perm(word, cb, 0x7652u), a3 = __byte_perm(word, cb, 0x7653u);
    return (lds_u32<(4 * W + 0) * 256>(a0) + lds_u32<(4 * W + 1) * 256>(a1)) +
           (lds_u32<(4 * W + 2) * 256>(a2) + lds_u32<(4 * W + 3) * 256>(a3));
}

struct LowPrep {
    float width, vl, half;
};

// Searcher::preparing for one (query, cluster) pair by all NT threads:
// residual r = q - c (kept in `res`), half = sum(r)/2 (16-lane order + tree),
// vl = min(0, min r), vr = max(0, max r), width = (vr - vl) / 16383,
// qq_i = (uint16)trunc((r_i - vl) * (float)(1/width) + 0.5), and the 6-dim
// tables of qq (32-bit, no offset).  red: >= 40 words.
template <int NT>
__device__ void low_prepare(const float* __restrict__ q, const float* __restrict__ c, int D,
                            float* res, uint32_t* qq, uint8_t* tab, float* red, LowPrep& out) {
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float mn = 0.f, mx = 0.f;  // data_range16 starts both from zero
    for (int i = tid; i < D; i += NT) {
        const float r = __fsub_rn(q[i], c[i]);
        res[i] = r;
        mn = fminf(mn, r);
        mx = fmaxf(mx, r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
        red[warp] = mn;
        red[8 + warp] = mx;
    }
    __syncthreads();
    float vl = red[0], vr = red[8];
#pragma unroll
    for (int w = 1; w < NW; ++w) {
        vl = fminf(vl, red[w]);
        vr = fmaxf(vr, red[8 + w]);
    }
    const float width = __fdiv_rn(__fsub_rn(vr, vl), 16383.f);
    const float oow = recip_via_double(width);
    const int nqq = hex_qq_len(D);
    for (int i = tid; i < nqq; i += NT) {
        uint32_t v = 0;
        if (i < D) {
            const float t = __fadd_rn(__fmul_rn(__fsub_rn(res[i], vl), oow), 0.5f);
            v = (uint32_t)__float2int_rz(t) & 0xffffu;  // cvttps then the low 16 bits
        }
        qq[i] = v;
    }
    if (warp == 0) {  // minus_sum16's sum: 16 ordered lanes + the reduce tree
        float acc = 0.f;
        if (lane < 16)
            for (int i = lane; i < D; i += 16) acc = __fadd_rn(acc, res[i]);
        const float s = tree16_sum(acc);
        if (lane == 0) red[16] = __fmul_rn(0.5f, s);
    }
    __syncthreads();
    const int ntask = hex_chunks(D) * 16 * 16;  // (table, 4 entries)
    for (int task = tid; task < ntask; task += NT) {
        const int t = task >> 4, m = task & 15;
        const uint32_t* qt = qq + kHexDims * t;
        uint32_t e[4];
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int idx = 4 * m + l;
            uint32_t s = 0;
#pragma unroll
            for (int j = 0; j < kHexDims; ++j) s += ((idx >> j) & 1) ? qt[j] : 0u;
            e[l] = s;
        }
        reinterpret_cast<uint4*>(tab + 256 * t)[m] = make_uint4(e[0], e[1], e[2], e[3]);
    }
    __syncthreads();
    out.width = width;
    out.vl = vl;
    out.half = red[16];
}

struct LowFactors {
    const float* x2;     // [blocks*32] ||o - c||^2
    const float* fip;    // [blocks*32] inner-product factor
    const float* sumxb;  // [blocks*32] set bits of the 1-bit code
    const float* ferr;   // [blocks*32] error factor
};

// rabitq_ip and the lower bound of one vector (Searcher.hpp:200-224).
__device__ __forceinline__ float low_lower_bound(int S, const LowPrep& p, float sqr_y, float y,
                                                 float x2, float fip, float sumxb, float ferr,
                                                 float& rabitq_ip) {
    float ip = __fadd_rn(__fmul_rn(__int2float_rn(S), p.width), __fmul_rn(sumxb, p.vl));
    ip = __fsub_rn(ip, p.half);
    rabitq_ip = ip;
    const float a = __fmul_rn(ip, fip);
    const float err = __fmul_rn(ferr, y);
    return __fsub_rn(__fadd_rn(x2, sqr_y), __fadd_rn(a, err));
}

struct LowScanArgs {
    const float* qrot;
    const float* centroids;
    const uint32_t* probe_cid;
    const float* probe_sqy;
    const uint8_t* codes;
    const uint32_t* c_first_block;
    const uint32_t* c_nblocks;
    const uint32_t* c_size;
    const uint64_t* s_off;
    int32_t* S;
    float* qp_width;   // [nq][nprobe]
    float* qp_vl;      // [nq][nprobe]
    float* qp_half;    // [nq][nprobe]
    float* bmin;       // optional: smallest lower bound per block (-inf when a lane's is NaN)
    LowFactors f;
    uint32_t* status;
    int D, nprobe;
};

// Shared memory: [pad to 256][tables][ring][residual D][qq][bars][red 64]
__host__ __device__ constexpr size_t low_scan_smem_bytes(int D) {
    return 256 + (size_t)low_table_bytes(D) + (size_t)kScanWarps * kRing * kUnitBytes + (size_t)D * 4 +
           (size_t)hex_qq_len(D) * 4 + (size_t)kScanWarps * kRing * 8 + 64 * 4;
}

// One block per (query, probed cluster), as scan_kernel.
__global__ void __launch_bounds__(kScanWarps * 32, 1) scan_lowacc_kernel(LowScanArgs a) {
    extern __shared__ uint8_t smem_raw[];
    const int D = a.D;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t raw_s = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = (256u - (raw_s & 255u)) & 255u;
    uint8_t* tables = smem_raw + pad;
    const uint32_t ring_off = pad + low_table_bytes(D);
    float* res = reinterpret_cast<float*>(smem_raw + ring_off + kScanWarps * kRing * kUnitBytes);
    uint32_t* qq = reinterpret_cast<uint32_t*>(res + D);
    const uint32_t bars_s = (uint32_t)__cvta_generic_to_shared(qq + hex_qq_len(D));
    float* red = reinterpret_cast<float*>(smem_raw + (bars_s - raw_s) + kScanWarps * kRing * 8);

    const uint32_t pair = blockIdx.x;
    const uint32_t q = pair / (uint32_t)a.nprobe;
    const uint32_t cid = a.probe_cid[pair];
    const uint32_t nb = a.c_nblocks[cid];
    const uint32_t fblock = a.c_first_block[cid];
    if (tid == 0) {
        for (int i = 0; i < kScanWarps * kRing; ++i) mbar_init(bars_s + 8 * i, 1);
        mbar_init_fence();
        reinterpret_cast<uint32_t*>(red)[40] = raw_s + pad;
    }
    __syncthreads();
    UnitStream us;
    us.block_bytes = code_block_bytes(D);
    us.codes = a.codes + (size_t)fblock * us.block_bytes;
    us.nc = hex_chunks(D);
    us.nu = (us.nc + kUnitChunks - 1) / kUnitChunks;
    us.b_first = warp;
    us.stride = kScanWarps;
    const uint32_t my_blocks = (uint32_t)warp < nb ? (nb - warp + kScanWarps - 1) / kScanWarps : 0u;
    us.total = my_blocks * us.nu;
    us.ring = raw_s + ring_off + warp * kRing * kUnitBytes;
    us.bars = bars_s + warp * kRing * 8;
    us.count = 0;
    if (lane == 0) us.issue_first();

    LowPrep pp;
    low_prepare<kScanWarps * 32>(a.qrot + (size_t)q * D, a.centroids + (size_t)cid * D, D, res, qq,
                                 tables, red, pp);
    if (tid == 0) {
        a.qp_width[pair] = pp.width;
        a.qp_vl[pair] = pp.vl;
        a.qp_half[pair] = pp.half;
    }
    const uint32_t tables_s = reinterpret_cast<volatile uint32_t*>(red)[40];
    const float sqr_y = a.probe_sqy[pair];
    const float y = __fsqrt_rn(sqr_y);
    const uint32_t csize = a.c_size[cid];
    int32_t* out = a.S + a.s_off[pair];

    uint32_t m = 0;
    bool ok = true;
    for (uint32_t n = 0; n < my_blocks && ok; ++n) {
        int acc = 0;
        for (uint32_t u = 0; u < us.nu; ++u, ++m) {
            if (!us.wait_next()) {
                ok = false;
                break;
            }
            const uint32_t st = us.stage_next() + lane * 16;
            const uint32_t c0 = u * kUnitChunks;
            const uint32_t nch = min((uint32_t)kUnitChunks, us.nc - c0);
#pragma unroll
            for (uint32_t cc = 0; cc < (uint32_t)kUnitChunks; ++cc) {
                if (cc < nch) {
                    const uint4 w = lds128(st + cc * 512);
                    const uint32_t cb = tables_s + (c0 + cc) * 4096;
                    acc += low_lookup4<0>(w.x, cb) + low_lookup4<1>(w.y, cb);
                    acc += low_lookup4<2>(w.z, cb) + low_lookup4<3>(w.w, cb);
                }
            }
            us.refill(m, lane);
            us.advance();
        }
        if (!ok) break;
        const uint32_t b = warp + n * kScanWarps;
        out[32 * b + lane] = acc;
        if (a.bmin) {
            const size_t v = (size_t)(fblock + b) * 32 + lane;
            float rip;
            const float lb = low_lower_bound(acc, pp, sqr_y, y, a.f.x2[v], a.f.fip[v], a.f.sumxb[v],
                                             a.f.ferr[v], rip);
            const bool valid = 32 * b + lane < csize;
            const bool nan = __any_sync(0xffffffffu, valid && lb != lb);
            const float mn = warp_min(valid ? lb : INFINITY);
            if (lane == 0) a.bmin[a.s_off[pair] / 32 + b] = nan ? -INFINITY : mn;
        }
    }
    if (!ok && lane == 0) {
        us.drain(m);
        if (a.status) atomicOr(a.status, kScanTimeoutBit);
    }
}

struct LowRefineArgs {
    const float* qrot;
    const float* centroids;
    const uint32_t* probe_cid;
    const float* probe_sqy;
    const uint64_t* s_off;
    const int32_t* S;
    const float* qp_width;
    const float* qp_vl;
    const float* qp_half;
    const float* bmin;
    LowFactors f;
    const uint8_t* excode;
    uint64_t ex_row;
    const float* xipnorm;
    const uint32_t* ids;
    const uint32_t* c_first_block;
    const uint32_t* c_first_vec;
    const uint32_t* c_size;
    uint32_t* out_ids;
    float* out_dists;
    int nq, D, EX, nprobe, k;
};

constexpr int kLowRefineWarps = 4;  // one query per warp

// Per warp and query: [residual D][pool_d kpad][pool_id kpad][ed 32][lb 32][cs 32]
__host__ __device__ constexpr size_t low_refine_smem_per_warp(int D, int kpad) {
    return (size_t)D * 4 + (size_t)kpad * 8 + 3 * 32 * 4;
}

// Searcher::search_cluster / scan_one_block for one query per warp: per
// block, the lanes whose lower bound is within the running threshold at the
// block's start (a superset) get their exact distances (8 quads at a time,
// the reference's IP_FUNC order on the residual); then the block is replayed
// lane by lane: a lane is offered to the pool when its lower bound is still
// <= the threshold, which is refreshed after every insertion.
template <int EX>
__global__ void __launch_bounds__(kLowRefineWarps * 32) refine_lowacc_kernel(LowRefineArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = blockIdx.x * kLowRefineWarps + warp;
    const int D = a.D, k = a.k, kpad = (k + 31) & ~31;
    uint8_t* base = smem_raw + (size_t)warp * low_refine_smem_per_warp(D, kpad);
    float* res = reinterpret_cast<float*>(base);
    float* pool_d = res + D;
    uint32_t* pool_id = reinterpret_cast<uint32_t*>(pool_d + kpad);
    float* ed_s = reinterpret_cast<float*>(pool_id + kpad);
    float* lb_s = ed_s + 32;
    float* cs = lb_s + 32;
    if (q >= a.nq) return;
    for (int i = lane; i < kpad; i += 32) {
        pool_d[i] = 0.f;
        pool_id[i] = 0u;
    }
    __syncwarp();
    int size = 0;
    float distk = FLT_MAX;
    const float facr = (float)(1 << EX), facr1 = (float)((1 << EX) - 1);
    const float* qv = a.qrot + (size_t)q * D;
    for (int p = 0; p < a.nprobe; ++p) {
        const size_t qp = (size_t)q * a.nprobe + p;
        const uint32_t cid = a.probe_cid[qp];
        const float sqr_y = a.probe_sqy[qp];
        const float y = __fsqrt_rn(sqr_y);
        LowPrep pp;
        pp.width = a.qp_width[qp];
        pp.vl = a.qp_vl[qp];
        pp.half = a.qp_half[qp];
        const uint32_t n = a.c_size[cid], fb = a.c_first_block[cid], fv = a.c_first_vec[cid];
        const int32_t* S = a.S + a.s_off[qp];
        const float* bmin = a.bmin ? a.bmin + a.s_off[qp] / 32 : nullptr;
        const float* cv = a.centroids + (size_t)cid * D;
        for (int i = lane; i < D; i += 32) res[i] = __fsub_rn(qv[i], cv[i]);
        __syncwarp();
        const float a_half = __fmul_rn(facr1, pp.half);
        for (uint32_t b = 0; b < (n + 31) / 32; ++b) {
            if (bmin && bmin[b] > distk) continue;  // no lane can pass now or later
            const bool valid = 32 * b + lane < n;
            const size_t vi = (size_t)(fb + b) * 32 + lane;
            float rip = 0.f, x2 = 0.f, lb = INFINITY;
            if (valid) {
                x2 = a.f.x2[vi];
                lb = low_lower_bound(S[32 * b + lane], pp, sqr_y, y, x2, a.f.fip[vi], a.f.sumxb[vi],
                                     a.f.ferr[vi], rip);
            }
            const bool sup = valid && !(lb > distk);
            uint32_t list = __ballot_sync(0xffffffffu, sup);
            if (!list) continue;
            lb_s[lane] = lb;
            // exact distances of the listed lanes, 8 quads at a time
            const int g = lane >> 2, r = lane & 3;
            for (uint32_t rest = list; rest;) {
                // the g-th listed lane of this round (quads past the end repeat the first)
                uint32_t mm = rest;
                int pick = __ffs(mm) - 1;
                for (int t = 0; t < g && mm; ++t) {
                    mm &= mm - 1;
                    if (mm) pick = __ffs(mm) - 1;
                }
                const bool mine = __popc(rest) > g;
                const size_t pos = (size_t)fv + 32 * b + pick;
                const uint4* row = reinterpret_cast<const uint4*>(a.excode + pos * a.ex_row);
                float ip[2];
                ex_ip_quad<ex_storage_bits(EX), 1>(reinterpret_cast<const float4*>(res), row, row, r,
                                                   D / 16, ip);
                const float ripj = __shfl_sync(0xffffffffu, rip, pick);
                const float x2j = __shfl_sync(0xffffffffu, x2, pick);
                if (mine && r == 0) {
                    const float inner = __fsub_rn(__fadd_rn(__fmul_rn(facr, ripj), ip[0]), a_half);
                    ed_s[pick] = __fsub_rn(__fadd_rn(x2j, sqr_y), __fmul_rn(__ldg(a.xipnorm + pos), inner));
                }
                for (int t = 0; t < 8 && rest; ++t) rest &= rest - 1;
            }
            __syncwarp();
            // replay: lanes in order against the threshold as it stands
            for (uint32_t mm = list; mm; mm &= mm - 1) {
                const int j = __ffs(mm) - 1;
                if (lb_s[j] > distk) continue;
                const float d = ed_s[j];
                const uint32_t id = __ldg(a.ids + (size_t)fv + 32 * b + j);
                pool_merge_block(pool_d, pool_id, size, k, distk, lane == j, d, id, cs, lane);
            }
        }
        __syncwarp();
    }
    uint32_t* oid = a.out_ids + (size_t)q * k;
    for (int i = lane; i < k; i += 32) {
        oid[i] = i < size ? pool_id[i] : 0u;
        if (a.out_dists) a.out_dists[(size_t)q * k + i] = i < size ? pool_d[i] : __int_as_float(0x7f800000);
    }
}

}  // namespace erq
