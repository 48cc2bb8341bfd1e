// Per-(query, probed cluster) preparation and the FastScan accumulation.
//
// For a (query q, probed cluster c) pair the reference computes
//   1. unit_q = (q_r - c) * (float)(1.0/y), max |unit_q|      normalize_query16,
//      data_range16               inc/utils/space.hpp:749-778, 608-628
//   2. delta = vmax / 8191, qq = round-half-away(unit_q / delta)
//                                 high_acc_quantize16, inc/utils/space.hpp:695-711
//   3. sumq = 16-lane ordered sum of unit_q (normalize_query16's return value)
//   4. S_v = <x_b(v), qq> for every vector v of the cluster, exact in int32:
//      4-dim lookup tables and u16 lanes plus a shift in the reference
//      (pack_high_acc_LUT, inc/index/HASearcher.hpp:128-185;
//      accumulate_one_block_high_acc, inc/index/fastscan/FastScan.hpp:214-308).
// S is an exact integer dot product, so any grouping of the dims gives the
// same S.  Here the dims go in groups of six (64-entry tables, D/6 lookups per
// vector where the reference's 4-dim tables take D/4):
//   table_t[e] = sum_{j in bits(e)} qq[6t + j] - vmin_t,
//   vmin_t = sum_j min(qq[6t + j], 0)      (so 0 <= table_t[e] <= 6 * 8191)
//   S_v = sum_t table_t[idx_t(v)] + sum_t vmin_t,
//   idx_t(v) = sum_j bit(v, 6t + j) << j   (dims >= D contribute 0 bits).
// A table is 64 u16 = 128 bytes = one row of the 32 shared-memory banks, so a
// warp whose 32 lanes (= the 32 vectors of a block) look up one table at once
// needs one wavefront whatever the indices.
//
// Device code layout (built by transform_blocks_kernel, layout.cuh): per
// 32-vector block, chunks of 16 groups; chunk k is 512 bytes, lane v's 16
// bytes at 16v, byte i = 2 * idx_{16k+i}(v) + 128 * (i & 1).  Tables of chunk
// k sit at a 256-aligned base + 2048k, table 16k + i at + 128i, so a byte
// permute that drops the code byte into the base's low byte gives the address
// of the entry, with (i >> 1) * 256 as the load's immediate offset.
//
// The codes reach shared memory by bulk asynchronous copies (cp.async.bulk,
// completion counted on an mbarrier): each warp owns a ring of kRing stages
// of kUnitChunks chunks and its lane 0 keeps kRing copies of the warp's next
// units in flight; the first copies are issued before the preparation, which
// hides their latency.  Lanes read their 16 code bytes of a chunk with one
// 128-bit shared load.
//
// S, delta and sumq go to global memory; the lower bound and the refinement
// that depend on the running top-k threshold happen in refine.cuh.
#pragma once

#include "common.cuh"
#include "mbarrier.cuh"

namespace erq {

constexpr int kHexDims = 6;
__host__ __device__ constexpr int hex_groups(int D) { return (D + kHexDims - 1) / kHexDims; }
__host__ __device__ constexpr int hex_chunks(int D) { return (hex_groups(D) + 15) / 16; }
// device bytes of one 32-vector block's codes
__host__ __device__ constexpr uint32_t code_block_bytes(int D) { return (uint32_t)hex_chunks(D) * 512u; }
// shared bytes of one query's tables
__host__ __device__ constexpr uint32_t hex_table_bytes(int D) { return (uint32_t)hex_chunks(D) * 2048u; }
// qq entries (padded with zeros to whole chunks)
__host__ __device__ constexpr int hex_qq_len(int D) { return hex_chunks(D) * 16 * kHexDims; }

constexpr int kUnitChunks = 4;                   // chunks per staged copy
constexpr uint32_t kUnitBytes = kUnitChunks * 512;
constexpr int kRing = 2;                         // staged copies per warp
constexpr uint32_t kScanWaitLimit = 1u << 24;    // polls before a wait gives up
constexpr uint32_t kScanDrainLimit = 1u << 26;   // polls of the exit drain
constexpr uint32_t kScanTimeoutBit = 2u;         // bit of the device status word

struct ScanArgs {
    const float* qrot;        // [nq][D] rotated queries
    const float* centroids;   // [K][D] rotated centroids
    const uint32_t* probe_cid; // [nq][nprobe]
    const float* probe_sqy;   // [nq][nprobe]
    const uint8_t* codes;     // device block layout (above)
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
    uint32_t* status;         // device status word (bit kScanTimeoutBit: a wait ran out)
    int D;
    int nprobe;
};

constexpr int kScanWarps = 8;

__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr));
    return v;
}
template <int OFF>
__device__ __forceinline__ int lds_u16(uint32_t addr) {
    int v;
    asm("ld.shared.u16 %0, [%1+%2];" : "=r"(v) : "r"(addr), "n"(OFF));
    return v;
}

// The 2 lookups of bytes K and K+1 of code word `word` (groups 4W+K, 4W+K+1
// of chunk base `cb`) for queries J..QB-1, tables QSTR bytes apart.
template <int W, int K, int J, int QB, int QSTR>
__device__ __forceinline__ void hex_pair(uint32_t word, uint32_t cb, int qn, int (&acc)[QB]) {
    if constexpr (J < QB) {
        const uint32_t a0 = __byte_perm(word, cb, 0x7650u | K);
        const uint32_t a1 = __byte_perm(word, cb, 0x7650u | (K + 1));
        constexpr int OFF = (2 * W + (K >> 1)) * 256 + J * QSTR;
        if (J == 0 || J < qn) acc[J] += lds_u16<OFF>(a0) + lds_u16<OFF>(a1);
        hex_pair<W, K, J + 1, QB, QSTR>(word, cb, qn, acc);
    }
}

// 16 lookups (one chunk) of one lane for the first qn of QB queries.
template <int QB, int QSTR>
__device__ __forceinline__ void hex_lookup16(uint4 w, uint32_t cb, int qn, int (&acc)[QB]) {
    hex_pair<0, 0, 0, QB, QSTR>(w.x, cb, qn, acc);
    hex_pair<0, 2, 0, QB, QSTR>(w.x, cb, qn, acc);
    hex_pair<1, 0, 0, QB, QSTR>(w.y, cb, qn, acc);
    hex_pair<1, 2, 0, QB, QSTR>(w.y, cb, qn, acc);
    hex_pair<2, 0, 0, QB, QSTR>(w.z, cb, qn, acc);
    hex_pair<2, 2, 0, QB, QSTR>(w.z, cb, qn, acc);
    hex_pair<3, 0, 0, QB, QSTR>(w.w, cb, qn, acc);
    hex_pair<3, 2, 0, QB, QSTR>(w.w, cb, qn, acc);
}

struct PairPrep {
    float delta, sumq;
    int shift;
};

// Steps 1-3 and the tables of one (query, cluster) pair, by all NT threads of
// the block (two block barriers).  unit_q: D floats; tab: hex_table_bytes(D)
// bytes, 256-aligned; red: at least 32 + NT / 32 words.  q, c: the rotated
// query and centroid.
template <int NT>
__device__ void hex_prepare(const float* __restrict__ q, const float* __restrict__ c, float sqy,
                            int D, float* unit_q, uint8_t* tab, float* red,
                            PairPrep& out) {
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float y = __fsqrt_rn(sqy);
    const bool normal = y > kNormEps;
    const float fac = normal ? recip_via_double(y) : 0.f;
    const float fill = recip_via_double(__fsqrt_rn((float)D));
    const float4* qv = reinterpret_cast<const float4*>(q);
    const float4* cv = reinterpret_cast<const float4*>(c);

    // 1. unit_q and max |unit_q|
    float vmax = 0.f;
    for (int g = tid; g < D / 4; g += NT) {
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
    for (int w = 1; w < NW; ++w) vmax = fmaxf(vmax, red[w]);
    const float delta = __fdiv_rn(vmax, 8191.f);

    // 2. tables, one thread per table, each quantizing its own six dims
    //    (qq = round-half-away(unit_q / delta), zero past D): entry 8m + l = H[m] + L[l] with
    //    L[l] = sum of q0..q2 over the bits of l minus their negative part and
    //    H[m] the same of q3..q5; the eight 16-byte rows go out in an order
    //    rotated by t, so the lanes of a warp store to distinct banks
    int vsum = 0;
    const int ntab = hex_chunks(D) * 16;
    for (int t = tid; t < ntab; t += NT) {
        int qt[kHexDims];
#pragma unroll
        for (int j = 0; j < kHexDims; ++j) {
            const int i = kHexDims * t + j;
            qt[j] = i < D ? (int)(int16_t)quantize_round(__fdiv_rn(unit_q[i], delta)) : 0;
        }
        const int q0 = qt[0], q1 = qt[1], q2 = qt[2], q3 = qt[3], q4 = qt[4], q5 = qt[5];
        const int vlo = min(q0, 0) + min(q1, 0) + min(q2, 0);
        const int vhi = min(q3, 0) + min(q4, 0) + min(q5, 0);
        const uint32_t l0 = (uint32_t)(-vlo), l1 = (uint32_t)(q0 - vlo), l2 = (uint32_t)(q1 - vlo);
        const uint32_t l3 = (uint32_t)(q0 + q1 - vlo), l4 = (uint32_t)(q2 - vlo);
        const uint32_t l5 = (uint32_t)(q0 + q2 - vlo), l6 = (uint32_t)(q1 + q2 - vlo);
        const uint32_t l7 = (uint32_t)(q0 + q1 + q2 - vlo);
        // two 16-bit entries per word; H + L < 2^16, so a 32-bit add never carries
        const uint32_t p0 = l0 | (l1 << 16), p1 = l2 | (l3 << 16), p2 = l4 | (l5 << 16),
                       p3 = l6 | (l7 << 16);
        uint4* row = reinterpret_cast<uint4*>(tab + 128 * t);
#pragma unroll
        for (int s8 = 0; s8 < 8; ++s8) {
            const int m = (s8 + t) & 7;
            const uint32_t h = (uint32_t)(((m & 1) ? q3 : 0) + ((m & 2) ? q4 : 0) + ((m & 4) ? q5 : 0) - vhi);
            const uint32_t hd = h * 0x10001u;
            row[m] = make_uint4(p0 + hd, p1 + hd, p2 + hd, p3 + hd);
        }
        vsum += vlo + vhi;
    }
    vsum = __reduce_add_sync(0xffffffffu, vsum);
    if (lane == 0) reinterpret_cast<int*>(red)[32 + warp] = vsum;
    // sumq (16 ordered chains + tree) on the last warp, which holds the
    // fewest tables when they do not fill the block
    if (warp == NW - 1) {
        float acc = 0.f;
        if (lane < 16) {
            // the chain's order is fixed; its loads are not: 8 at a time ahead of the adds
            int i = lane;
            for (; i + 7 * 16 < D; i += 8 * 16) {
                float v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = unit_q[i + 16 * u];
#pragma unroll
                for (int u = 0; u < 8; ++u) acc = __fadd_rn(acc, v[u]);
            }
            for (; i < D; i += 16) acc = __fadd_rn(acc, unit_q[i]);
        }
        const float s = tree16_sum(acc);
        if (lane == 0) red[NW] = normal ? s : __fmul_rn((float)D, fill);
    }
    __syncthreads();
    // every red word read below was written before the barrier above, and the
    // next call writes them only after its first barrier, which these reads precede
    int shift = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) shift += reinterpret_cast<const int*>(red)[32 + w];
    out.delta = delta;
    out.sumq = red[NW];
    out.shift = shift;
}

// One warp's stream of staged code units for one cluster (or chunk of it):
// blocks b_first, b_first + stride, ... , each cut into units of up to
// kUnitChunks chunks; `total` units in all.  Units m < min(total, c + kRing)
// are issued once c units are consumed.  `count` is the warp's running number
// of units of earlier streams, which fixes each unit's ring slot and barrier
// phase across items.
struct UnitStream {
    const uint8_t* codes;   // the cluster's first block
    uint32_t block_bytes, nc, nu;  // bytes per block, chunks per block, units per block
    uint32_t b_first, stride, total;  // first block, block step, units in the stream
    uint32_t ring, bars;    // this warp's stages and full barriers (shared addresses)
    uint32_t count;         // units of earlier streams of this warp

    __device__ __forceinline__ void issue(uint32_t m) const {  // lane 0 only
        const uint32_t n = m / nu, u = m - n * nu;
        const uint32_t nch = min((uint32_t)kUnitChunks, nc - u * kUnitChunks);
        const uint32_t slot = (count + m) % kRing;
        const uint8_t* src = codes + (size_t)(b_first + n * stride) * block_bytes + u * kUnitBytes;
        mbar_expect_tx(bars + 8 * slot, nch * 512);
        bulk_g2s(ring + slot * kUnitBytes, src, nch * 512, bars + 8 * slot);
    }
    __device__ __forceinline__ void issue_first() const {  // lane 0 only
        for (uint32_t m = 0; m < total && m < (uint32_t)kRing; ++m) issue(m);
    }
    // after unit m is consumed by the whole warp (lane 0 issues, all lanes call)
    __device__ __forceinline__ void refill(uint32_t m, int lane) const {
        __syncwarp();
        if (lane == 0 && m + kRing < total) {
            fence_proxy_async_smem();  // the warp's reads of the slot before the copy's writes
            issue(m + kRing);
        }
    }
    // The consumer's cursor: ring slot and barrier parity of the next unit
    // (count + m); advance() after each consumed unit.
    uint32_t slot = 0, phase = 0;
    __device__ __forceinline__ void advance() {
        if (++slot == (uint32_t)kRing) {
            slot = 0;
            phase ^= 1u;
        }
    }
    // all lanes; false (warp-uniform) if the next unit's copy did not land in time
    __device__ __forceinline__ bool wait_next() const {
        return __all_sync(0xffffffffu, mbar_wait(bars + 8 * slot, phase, kScanWaitLimit));
    }
    __device__ __forceinline__ uint32_t stage_next() const { return ring + slot * kUnitBytes; }
    // lane 0, after a wait gave up at unit `consumed`: lets every copy issued
    // but not consumed land before the block exits or reuses the ring
    __device__ __forceinline__ void drain(uint32_t consumed) const {
        const uint32_t issued = min(total, consumed + (uint32_t)kRing);
        for (uint32_t m = consumed; m < issued; ++m) {
            const uint32_t slot = (count + m) % kRing, parity = ((count + m) / kRing) & 1;
            mbar_wait(bars + 8 * slot, parity, kScanDrainLimit);
        }
    }
};

// Shared memory of scan_kernel: [pad to 256][tables][ring][unit_q][bars][red 64]
__host__ __device__ constexpr size_t scan_smem_bytes(int D) {
    return 256 + (size_t)hex_table_bytes(D) + (size_t)kScanWarps * kRing * kUnitBytes +
           (size_t)D * 4 + (size_t)kScanWarps * kRing * 8 + 64 * 4;
}

__global__ void __launch_bounds__(kScanWarps * 32, 2) scan_kernel(ScanArgs a) {
    extern __shared__ uint8_t smem_raw[];
    const int D = a.D;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const uint32_t raw_s = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = (256u - (raw_s & 255u)) & 255u;
    uint8_t* tables = smem_raw + pad;
    const uint32_t ring_off = pad + hex_table_bytes(D);
    float* unit_q = reinterpret_cast<float*>(smem_raw + ring_off + kScanWarps * kRing * kUnitBytes);
    const uint32_t bars_s = (uint32_t)__cvta_generic_to_shared(unit_q + D);
    float* red = reinterpret_cast<float*>(smem_raw + (bars_s - raw_s) + kScanWarps * kRing * 8);

    const uint32_t pair = a.order ? a.order[blockIdx.x] : blockIdx.x;
    const uint32_t q = pair / (uint32_t)a.nprobe;
    if (a.q_nprobe && (int)(pair - q * (uint32_t)a.nprobe) >= a.q_nprobe[q]) return;
    const uint32_t cid = a.probe_cid[pair];
    const uint32_t nb = a.c_nblocks[cid];
    const uint32_t fblock = a.c_first_block[cid];

    if (tid == 0) {
        for (int i = 0; i < kScanWarps * kRing; ++i) mbar_init(bars_s + 8 * i, 1);
        mbar_init_fence();
        reinterpret_cast<uint32_t*>(red)[40] = raw_s + pad;  // tables, read back below
    }
    __syncthreads();

    // this warp's blocks: warp, warp + kScanWarps, ...; first copies now
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

    PairPrep pp;
    hex_prepare<kScanWarps * 32>(a.qrot + (size_t)q * D, a.centroids + (size_t)cid * D,
                                 a.probe_sqy[pair], D, unit_q, tables, red, pp);
    if (tid == 0) {
        a.qp_sumq[pair] = pp.sumq;
        a.qp_delta[pair] = pp.delta;
    }
    // The lookups are inline PTX; their addresses derive from this shared read,
    // which cannot move above the barriers of hex_prepare.
    static_assert(32 + kScanWarps <= 40, "hex_prepare's per-warp sums end below red[40]");
    const uint32_t tables_s = reinterpret_cast<volatile uint32_t*>(red)[40];
    const float y = __fsqrt_rn(a.probe_sqy[pair]);
    const LbConsts lbk = lb_consts(pp.sumq, y, recip_via_double(__fsqrt_rn((float)D)));
    const uint32_t csize = a.c_size[cid];
    int32_t* out = a.S + a.s_off[pair];

    uint32_t m = 0;
    bool ok = true;
    const uint32_t full_units = us.nc / kUnitChunks;  // units of kUnitChunks chunks per block
    for (uint32_t n = 0; n < my_blocks && ok; ++n) {
        int acc[1] = {0};
        for (uint32_t u = 0; u < us.nu; ++u, ++m) {
            if (!us.wait_next()) {
                ok = false;
                break;
            }
            const uint32_t st = us.stage_next() + lane * 16;
            const uint32_t cb = tables_s + u * (kUnitChunks * 2048);
            if (u < full_units) {
#pragma unroll
                for (uint32_t cc = 0; cc < (uint32_t)kUnitChunks; ++cc)
                    hex_lookup16<1, 0>(lds128(st + cc * 512), cb + cc * 2048, 1, acc);
            } else {
                for (uint32_t cc = 0; cc < us.nc - u * kUnitChunks; ++cc)
                    hex_lookup16<1, 0>(lds128(st + cc * 512), cb + cc * 2048, 1, acc);
            }
            us.refill(m, lane);
            us.advance();
        }
        if (!ok) break;
        const uint32_t b = warp + n * kScanWarps;
        const int sv = acc[0] + pp.shift;
        out[32 * b + lane] = sv;
        if (a.bmin) {
            const float on = a.onorm[(size_t)(fblock + b) * 32 + lane];
            const float lb = lower_bound(__fmul_rn(__int2float_rn(sv), pp.delta), on, lbk);
            const float mn = warp_min(32 * b + lane < csize ? lb : INFINITY);
            if (lane == 0) a.bmin[a.s_off[pair] / 32 + b] = mn;
        }
    }
    if (!ok && lane == 0) {
        us.drain(m);
        if (a.status) atomicOr(a.status, kScanTimeoutBit);
    }
}

}  // namespace erq
