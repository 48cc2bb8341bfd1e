// Batched FastScan over a (query block x cluster chunk) work list.
//
// The (query, probe) pairs of a batch are sorted by cluster (order.cuh).  A
// work item is one cluster c, up to QB of the pairs that probe c, and a chunk
// of up to CB of c's 32-vector blocks, so clusters of very uneven size
// (a few vectors to tens of thousands) split into items of bounded work.  A
// persistent kernel (a grid sized to the SMs) pulls items from a counter; the
// item count lives in device memory, so the launch needs no host sync and the
// whole search can be captured in a CUDA graph.
//
// Per item the QB lookup tables are built in shared memory exactly as in
// scan.cuh (same unit_q, delta, quantisation and entries), at a fixed stride
// of kQStride bytes per query.  A code word's table addresses are formed once
// and read for every query of the item with immediate offsets j * kQStride,
// so the shift / mask / permute work is shared by the QB queries.  S, delta
// and sumq land where the per-pair kernel puts them: every stage downstream is
// unchanged and the sums are bit-identical.
#pragma once

#include "common.cuh"
#include "scan.cuh"

namespace erq {

constexpr int kQStride = 16384;  // table bytes per query: 32 chunks of 512 (D <= 2048)

struct ScanBatchArgs {
    const float* qrot;
    const float* centroids;
    const uint32_t* probe_cid;     // [nq][nprobe]
    const float* probe_sqy;
    const uint8_t* codes;
    const uint32_t* c_first_block;
    const uint32_t* c_nblocks;
    const uint64_t* s_off;
    int32_t* S;
    float* qp_delta;
    float* qp_sumq;
    const float* onorm;            // [blocks*32] (for the block minima)
    const uint32_t* c_size;        // [K]
    float* bmin;                   // optional: smallest lower bound per scanned block
    const uint32_t* order_pairs;   // pairs sorted by cluster
    const uint32_t* bucket_end;    // [K + 1]: end of cluster c's run in order_pairs
    const uint32_t* item_off;      // [K + 1]: first item of cluster c; [K] = item count
    uint32_t* item_counter;        // zeroed before the launch
    int K, D, nprobe, CB;
};

// items of cluster c: ceil(m_c / QB) query blocks x max(1, ceil(nb_c / CB))
// chunks (an empty cluster still gets one item: its pairs need delta, sumq).
__global__ void scan_items_count_kernel(const uint32_t* __restrict__ bucket_end,
                                        const uint32_t* __restrict__ c_nblocks, int K, int QB, int CB,
                                        uint32_t* __restrict__ item_off) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) item_off[K] = 0;
    if (c >= K) return;
    const uint32_t m = bucket_end[c] - (c ? bucket_end[c - 1] : 0u);
    const uint32_t nch = max(1u, (c_nblocks[c] + CB - 1) / CB);
    item_off[c] = m ? ((m + QB - 1) / QB) * nch : 0u;
}

template <int OFF>
__device__ __forceinline__ int lds_s16_imm(uint32_t addr) {
    int v;
    asm volatile("ld.shared.s16 %0, [%1+%2];" : "=r"(v) : "r"(addr), "n"(OFF));
    return v;
}

// Lookups of one table address for queries J..QB-1 of the item (immediate
// offsets J * kQStride).
template <int J, int QB, bool kWindow1>
__device__ __forceinline__ void lookup_q(uint32_t a, uint32_t b, int qn, int (&acc_lo)[QB],
                                         int (&acc_hi)[QB]) {
    if constexpr (J < QB) {
        if (J < qn) {
            acc_lo[J] += lds_s16_imm<J * kQStride + (kWindow1 ? 256 : 0)>(a);
            acc_hi[J] += lds_s16_imm<J * kQStride + (kWindow1 ? 256 : 0)>(b);
        }
        lookup_q<J + 1, QB, kWindow1>(a, b, qn, acc_lo, acc_hi);
    }
}

// 8 lookups of one code word for each of the item's queries.
template <int QB, bool kWindow1>
__device__ __forceinline__ void lookup4_q(uint32_t lo2, uint32_t hi2, uint32_t base, int qn,
                                          int (&acc_lo)[QB], int (&acc_hi)[QB]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const uint32_t a = __byte_perm(lo2, base, 0x7650u | u);
        const uint32_t b = __byte_perm(hi2, base, 0x7650u | u);
        lookup_q<0, QB, kWindow1>(a, b, qn, acc_lo, acc_hi);
    }
}

// Shared memory: [pad to 256][QB tables of kQStride][unit_q D floats]
// [red 32 floats][item fields 4][per-query delta and lower-bound constants]
__host__ __device__ constexpr size_t scan_batch_smem_bytes(int QB, int D) {
    return 256 + (size_t)QB * kQStride + (size_t)D * 4 + 128 * 4;
}

template <int QB, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) scan_batched_kernel(ScanBatchArgs a) {
    extern __shared__ uint8_t smem_raw[];
    const int D = a.D;
    const int nchunk = D >> 6;
    const int ngroup = D >> 2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t raw_s = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = (256u - (raw_s & 255u)) & 255u;
    uint8_t* tables = smem_raw + pad;
    const uint32_t tables_s = raw_s + pad;
    float* unit_q = reinterpret_cast<float*>(tables + QB * kQStride);
    float* red = unit_q + D;                                    // [WARPS] maxima
    uint32_t* info = reinterpret_cast<uint32_t*>(red + 32);     // item fields
    float* jk = reinterpret_cast<float*>(info + 4);             // [QB][4]: delta, c1, c2, c3
    const float one_over_sqrtD = recip_via_double(__fsqrt_rn((float)D));
    const float fill = recip_via_double(__fsqrt_rn((float)D));
    const uint32_t h = lane >> 4, j16 = lane & 15;
    const uint32_t kconst = 0xC0804000u | (h ? 0x20202020u : 0u);
    const uint32_t vout = ((j16 & 1) ? (j16 >> 1) + 8 : (j16 >> 1)) + 16 * h;
    const uint32_t total = a.item_off[a.K];

    while (true) {
        if (tid == 0) {
            const uint32_t it = atomicAdd(a.item_counter, 1u);
            uint32_t c = 0;
            if (it < total) {
                // last cluster whose first item <= it
                int lo = 0, hi = a.K - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (a.item_off[mid] <= it) lo = mid; else hi = mid - 1;
                }
                c = (uint32_t)lo;
                // skip clusters with no items that share the same offset
                while (c + 1 < (uint32_t)a.K && a.item_off[c + 1] <= it) ++c;
            }
            info[0] = it;
            info[1] = c;
        }
        __syncthreads();
        const uint32_t it = info[0];
        if (it >= total) break;
        const uint32_t c = info[1];
        const uint32_t start = c ? a.bucket_end[c - 1] : 0u;
        const uint32_t m = a.bucket_end[c] - start;
        const uint32_t nb = a.c_nblocks[c];
        const uint32_t nch = max(1u, (nb + a.CB - 1) / a.CB);
        const uint32_t local = it - a.item_off[c];
        const uint32_t qblk = local / nch, chunk = local - qblk * nch;
        const uint32_t p0 = start + qblk * QB;
        const int qn = (int)min((uint32_t)QB, m - qblk * QB);
        const uint32_t b0 = chunk * a.CB, b1 = min(nb, b0 + a.CB);

        // tables of the item's queries (scan.cuh steps 1-4)
        uint32_t pairs[QB];
#pragma unroll
        for (int j = 0; j < QB; ++j) pairs[j] = j < qn ? a.order_pairs[p0 + j] : 0u;
        for (int j = 0; j < qn; ++j) {
            const uint32_t pair = a.order_pairs[p0 + j];
            const uint32_t q = pair / (uint32_t)a.nprobe;
            const float sqy = a.probe_sqy[pair];
            const float y = __fsqrt_rn(sqy);
            const bool normal = y > kNormEps;
            const float fac = normal ? recip_via_double(y) : 0.f;
            const float4* qv = reinterpret_cast<const float4*>(a.qrot + (size_t)q * D);
            const float4* cv = reinterpret_cast<const float4*>(a.centroids + (size_t)c * D);
            float vmax = 0.f;
            for (int g = tid; g < ngroup; g += blockDim.x) {
                float4 u;
                if (normal) {
                    const float4 x = qv[g], cc = cv[g];
                    u.x = __fmul_rn(__fsub_rn(x.x, cc.x), fac);
                    u.y = __fmul_rn(__fsub_rn(x.y, cc.y), fac);
                    u.z = __fmul_rn(__fsub_rn(x.z, cc.z), fac);
                    u.w = __fmul_rn(__fsub_rn(x.w, cc.w), fac);
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
            for (int w = 1; w < WARPS; ++w) vmax = fmaxf(vmax, red[w]);
            const float delta = __fdiv_rn(vmax, 8191.f);
            if (warp == 0) {
                float acc = 0.f;
                if (lane < 16)
                    for (int i = lane; i < D; i += 16) acc = __fadd_rn(acc, unit_q[i]);
                const float s = tree16_sum(acc);
                if (lane == 0) {
                    const float sq = normal ? s : __fmul_rn((float)D, fill);
                    if (chunk == 0) {
                        a.qp_sumq[pair] = sq;
                        a.qp_delta[pair] = delta;
                    }
                    const LbConsts k = lb_consts(sq, y, one_over_sqrtD);
                    jk[4 * j + 0] = delta;
                    jk[4 * j + 1] = k.c1;
                    jk[4 * j + 2] = k.c2;
                    jk[4 * j + 3] = k.c3;
                }
            }
            uint8_t* tj = tables + j * kQStride;
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
                    const int v1 = v0 + x3;
                    packed[e >> 1] = ((uint32_t)v0 & 0xffffu) | ((uint32_t)v1 << 16);
                }
                const int cc = g >> 4, w = g & 15, hh = w >> 3, u8 = w & 7;
                uint4* dst = reinterpret_cast<uint4*>(tj + cc * 512 + (u8 >> 2) * 256 + (u8 & 3) * 64 +
                                                      hh * 32);
                dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
                dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
            }
            __syncthreads();  // unit_q is rebuilt for the next query
        }
        if (tid == 0) info[2] = tables_s;
        __syncthreads();
        // lookups below are inline PTX whose addresses derive from this read
        const uint32_t tables_base = reinterpret_cast<volatile uint32_t*>(info)[2];

        const uint8_t* cl_codes = a.codes + (size_t)a.c_first_block[c] * (4 * D);
        for (uint32_t b = b0 + warp; b < b1; b += WARPS) {
            const uint2* src = reinterpret_cast<const uint2*>(cl_codes + (size_t)b * (4 * D)) + lane;
            int acc_lo[QB], acc_hi[QB];
#pragma unroll
            for (int j = 0; j < QB; ++j) acc_lo[j] = acc_hi[j] = 0;
#pragma unroll 2
            for (int ck = 0; ck < nchunk; ++ck) {
                const uint2 w = __ldg(src + ck * 32);
                const uint32_t base = tables_base + ck * 512;
                const uint32_t lo0 = ((w.x << 1) & 0x1E1E1E1Eu) | kconst;
                const uint32_t hi0 = ((w.x >> 3) & 0x1E1E1E1Eu) | kconst;
                lookup4_q<QB, false>(lo0, hi0, base, qn, acc_lo, acc_hi);
                const uint32_t lo1 = ((w.y << 1) & 0x1E1E1E1Eu) | kconst;
                const uint32_t hi1 = ((w.y >> 3) & 0x1E1E1E1Eu) | kconst;
                lookup4_q<QB, true>(lo1, hi1, base, qn, acc_lo, acc_hi);
            }
            const float on = a.bmin ? a.onorm[(size_t)(a.c_first_block[c] + b) * 32 + vout] : 0.f;
            const bool valid = 32 * b + vout < a.c_size[c];
#pragma unroll
            for (int j = 0; j < QB; ++j) {
                if (j < qn) {
                    int lo = acc_lo[j] + __shfl_xor_sync(0xffffffffu, acc_lo[j], 16);
                    int hi = acc_hi[j] + __shfl_xor_sync(0xffffffffu, acc_hi[j], 16);
                    const int sv = h ? hi : lo;
                    a.S[a.s_off[pairs[j]] + 32 * b + vout] = sv;
                    if (a.bmin) {
                        LbConsts k;
                        k.c1 = jk[4 * j + 1];
                        k.c2 = jk[4 * j + 2];
                        k.c3 = jk[4 * j + 3];
                        const float lb = lower_bound(__fmul_rn(__int2float_rn(sv), jk[4 * j]), on, k);
                        const float m = warp_min(valid ? lb : INFINITY);
                        if (lane == 0) a.bmin[a.s_off[pairs[j]] / 32 + b] = m;
                    }
                }
            }
        }
        __syncthreads();  // tables and info are reused by the next item
    }
}

}  // namespace erq
