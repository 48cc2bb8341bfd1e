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
// Per item each warp first starts the bulk copies of its first code units
// (scan.cuh: per-warp rings, cp.async.bulk + mbarriers), then the block
// builds the QB queries' 6-dim tables exactly as scan_kernel does, at a fixed
// stride of QSTR bytes per query, while the copies land.  A code byte's table
// address is formed once (one byte permute) and read for every query of the
// item with immediate offsets j * QSTR.  The last warp, which takes the
// fewest of an item's blocks, claims the next item and reads its cluster,
// pairs and sqy while the other warps finish, so a new item starts with its
// copies and table loads at once.  S, delta and sumq land where the
// per-pair kernel puts them: every stage downstream is unchanged and the sums
// are bit-identical.
#pragma once

#include "common.cuh"
#include "scan.cuh"

namespace erq {

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
    const uint32_t* c_order;       // [K]: the clusters in the order their items run
    const uint32_t* item_off;      // [K + 1]: first item of c_order[j]; [K] = item count
    uint32_t* item_counter;        // zeroed before the launch
    uint32_t* status;              // device status word (bit kScanTimeoutBit)
    int K, D, nprobe, CB;
};

// items of the j-th cluster c of c_order: ceil(m_c / QB) query blocks x
// max(1, ceil(nb_c / CB)) chunks (an empty cluster still gets one item: its
// pairs need delta, sumq; none when no pair probes c).  The clusters go
// largest first, so the work list ends with short items and the persistent
// blocks finish together.
__global__ void scan_items_count_kernel(const uint32_t* __restrict__ bucket_end,
                                        const uint32_t* __restrict__ c_nblocks,
                                        const uint32_t* __restrict__ c_order, int K, int QB, int CB,
                                        uint32_t* __restrict__ item_off) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0) item_off[K] = 0;
    if (j >= K) return;
    const uint32_t c = c_order[j];
    const uint32_t m = bucket_end[c] - (c ? bucket_end[c - 1] : 0u);
    const uint32_t nch = max(1u, (c_nblocks[c] + CB - 1) / CB);
    item_off[j] = m ? ((m + QB - 1) / QB) * nch : 0u;
}

// The position in c_order of the cluster that owns item `it` (it <
// item_off[K]): the last j in [0, K) with item_off[j] <= it (a cluster without
// items shares its successor's offset, so the last one is the owner).  A
// 32-way search by one warp: each round every lane tests one split point of
// the range, so K = 4096 takes 3 dependent loads where a binary search takes 12.
__device__ __forceinline__ uint32_t item_cluster(const uint32_t* __restrict__ item_off, int K,
                                                 uint32_t it, int lane) {
    int lo = 0, n = K;  // invariant: item_off[lo] <= it; the owner lies in [lo, lo + n)
    while (n > 1) {
        const int step = (n + 31) >> 5;
        const int idx = lo + lane * step;
        const bool le = idx < lo + n && item_off[idx] <= it;
        // item_off is non-decreasing, so the set lanes are a prefix (lane 0 always)
        const uint32_t bal = __ballot_sync(0xffffffffu, le);
        const int nlo = lo + (31 - __clz(bal)) * step;
        n = min(step, lo + n - nlo);
        lo = nlo;
    }
    return (uint32_t)lo;
}

// Words of the next-item record in shared memory (written by one warp):
// [0] item, [1] cluster, [2] first pair of the cluster's run, [3] pairs in
// the run, [4] blocks, [5] the cluster's first item, [6] its first block,
// [7] unused, then the item's pairs [QB] and their probe_sqy [QB] (zero past
// the item's last query).
__host__ __device__ constexpr int scan_item_words(int QB) { return 8 + 2 * QB; }

// Claims the next work item and reads everything the block needs to start it
// (cluster, run, blocks, pairs, sqy) into `nx`, by one whole warp.  Run by
// the warp with the fewest blocks while the others finish the current item,
// so these dependent loads stay off the item's critical path.
template <int QB>
__device__ __forceinline__ void claim_item(const ScanBatchArgs& a, uint32_t total, uint32_t* nx,
                                           int lane) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(a.item_counter, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it < total) {
        const uint32_t j = item_cluster(a.item_off, a.K, it, lane);
        const uint32_t c = a.c_order[j];
        const uint32_t start = c ? a.bucket_end[c - 1] : 0u;
        const uint32_t m_c = a.bucket_end[c] - start;
        const uint32_t nb = a.c_nblocks[c];
        const uint32_t ioff = a.item_off[j];
        const uint32_t fblock = a.c_first_block[c];
        const uint32_t nch = max(1u, (nb + a.CB - 1) / a.CB);
        const uint32_t qblk = (it - ioff) / nch;
        const uint32_t qn = min((uint32_t)QB, m_c - qblk * QB);
        if (lane < QB) {
            uint32_t pair = 0;
            float sqy = 0.f;
            if ((uint32_t)lane < qn) {
                pair = a.order_pairs[start + qblk * QB + lane];
                sqy = a.probe_sqy[pair];
            }
            nx[8 + lane] = pair;
            reinterpret_cast<float*>(nx)[8 + QB + lane] = sqy;
        }
        if (lane == 0) {
            nx[1] = c;
            nx[2] = start;
            nx[3] = m_c;
            nx[4] = nb;
            nx[5] = ioff;
            nx[6] = fblock;
        }
    }
    if (lane == 0) nx[0] = it;
}

// Table bytes per query slot of the batched kernel: the classes of padded
// dimension the kernels are built for.
__host__ __device__ constexpr int scan_qstride(int D) {
    return D <= 768 ? 16384 : (D <= 1536 ? 32768 : 45056);
}

// Shared memory: [pad to 256][QB tables, QSTR apart][ring][unit_q][bars]
// [red 64 words][4 words: table address][per-query delta, lower-bound
// constants, shift][next-item record]
__host__ __device__ constexpr size_t scan_batch_smem_bytes(int QB, int W, int QSTR, int D) {
    return 256 + (size_t)(QB == 1 ? (int)hex_table_bytes(D) : QB * QSTR) +
           (size_t)W * kRing * kUnitBytes + (size_t)D * 4 + (size_t)W * kRing * 8 + 64 * 4 + 4 * 4 + (size_t)QB * 8 * 4 +
           (size_t)scan_item_words(QB) * 4;
}

template <int QB, int WARPS, int QSTR>
__global__ void __launch_bounds__(WARPS * 32) scan_batched_kernel(ScanBatchArgs a) {
    extern __shared__ uint8_t smem_raw[];
    const int D = a.D;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t raw_s = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = (256u - (raw_s & 255u)) & 255u;
    const uint32_t tstride = QB == 1 ? hex_table_bytes(D) : (uint32_t)QSTR;
    uint8_t* tables = smem_raw + pad;
    const uint32_t ring_off = pad + QB * tstride;
    float* unit_q = reinterpret_cast<float*>(smem_raw + ring_off + WARPS * kRing * kUnitBytes);
    const uint32_t bars_s = (uint32_t)__cvta_generic_to_shared(unit_q + D);
    float* red = reinterpret_cast<float*>(smem_raw + (bars_s - raw_s) + WARPS * kRing * 8);
    uint32_t* info = reinterpret_cast<uint32_t*>(red + 64);     // [2]: the tables' address
    float* jk = reinterpret_cast<float*>(info + 4);             // [QB][8]: delta, c1, c2, c3, shift
    uint32_t* nx = reinterpret_cast<uint32_t*>(jk + QB * 8);    // next-item record
    const float one_over_sqrtD = recip_via_double(__fsqrt_rn((float)D));
    const uint32_t total = a.item_off[a.K];

    constexpr int kClaimWarp = WARPS - 1;  // takes the fewest blocks of every item
    if (tid == 0) {
        for (int i = 0; i < WARPS * kRing; ++i) mbar_init(bars_s + 8 * i, 1);
        mbar_init_fence();
        info[2] = raw_s + pad;
    }
    if (warp == kClaimWarp) claim_item<QB>(a, total, nx, lane);
    __syncthreads();

    UnitStream us;
    us.block_bytes = code_block_bytes(D);
    us.nc = hex_chunks(D);
    us.nu = (us.nc + kUnitChunks - 1) / kUnitChunks;
    us.stride = WARPS;
    us.ring = raw_s + ring_off + warp * kRing * kUnitBytes;
    us.bars = bars_s + warp * kRing * 8;
    us.count = 0;
    us.total = 0;
    us.slot = 0;
    us.phase = 0;
    bool ok = true;

    while (true) {
        // the item claimed during the previous one (or before the loop); every
        // read of the record comes before the block barrier that precedes the
        // claiming warp's next write
        const uint32_t it = nx[0];
        if (it >= total) break;
        const uint32_t c = nx[1];
        const uint32_t m_c = nx[3];
        const uint32_t nb = nx[4];
        const uint32_t nch = max(1u, (nb + a.CB - 1) / a.CB);
        const uint32_t local = it - nx[5];
        const uint32_t qblk = local / nch, chunk = local - qblk * nch;
        const int qn = (int)min((uint32_t)QB, m_c - qblk * QB);
        const uint32_t b0 = chunk * a.CB, b1 = min(nb, b0 + a.CB);
        const uint32_t fblock = nx[6];

        // this warp's blocks of the item: b0 + warp, b0 + warp + WARPS, ...
        us.count += us.total;
        us.codes = a.codes + (size_t)fblock * us.block_bytes;
        us.b_first = b0 + warp;
        const uint32_t my_blocks = us.b_first < b1 ? (b1 - us.b_first + WARPS - 1) / WARPS : 0u;
        us.total = ok ? my_blocks * us.nu : 0u;
        if (lane == 0) us.issue_first();

        // tables of the item's queries (scan.cuh)
        uint32_t pairs[QB];
#pragma unroll
        for (int j = 0; j < QB; ++j) pairs[j] = nx[8 + j];
        for (int j = 0; j < qn; ++j) {
            const uint32_t pair = nx[8 + j];
            const uint32_t q = pair / (uint32_t)a.nprobe;
            const float sqy = reinterpret_cast<const float*>(nx)[8 + QB + j];
            PairPrep pp;
            hex_prepare<WARPS * 32>(a.qrot + (size_t)q * D, a.centroids + (size_t)c * D, sqy, D,
                                    unit_q, tables + j * tstride, red, pp);
            if (tid == 0) {
                if (chunk == 0) {
                    a.qp_sumq[pair] = pp.sumq;
                    a.qp_delta[pair] = pp.delta;
                }
                const LbConsts k = lb_consts(pp.sumq, __fsqrt_rn(sqy), one_over_sqrtD);
                jk[8 * j + 0] = pp.delta;
                jk[8 * j + 1] = k.c1;
                jk[8 * j + 2] = k.c2;
                jk[8 * j + 3] = k.c3;
                reinterpret_cast<int*>(jk)[8 * j + 4] = pp.shift;
            }
        }
        __syncthreads();  // jk
        // lookups below are inline PTX whose addresses derive from this read
        const uint32_t tables_s = reinterpret_cast<volatile uint32_t*>(info)[2];

        uint32_t m = 0;
        const uint32_t full_units = us.nc / kUnitChunks;
        for (uint32_t n = 0; n < my_blocks && ok; ++n) {
            int acc[QB];
#pragma unroll
            for (int j = 0; j < QB; ++j) acc[j] = 0;
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
                        hex_lookup16<QB, QSTR>(lds128(st + cc * 512), cb + cc * 2048, qn, acc);
                } else {
                    for (uint32_t cc = 0; cc < us.nc - u * kUnitChunks; ++cc)
                        hex_lookup16<QB, QSTR>(lds128(st + cc * 512), cb + cc * 2048, qn, acc);
                }
                us.refill(m, lane);
                us.advance();
            }
            if (!ok) break;
            const uint32_t b = us.b_first + n * WARPS;
            const float on = a.bmin ? a.onorm[(size_t)(fblock + b) * 32 + lane] : 0.f;
            const bool valid = 32 * b + lane < a.c_size[c];
#pragma unroll
            for (int j = 0; j < QB; ++j) {
                if (j < qn) {
                    const int sv = acc[j] + reinterpret_cast<const int*>(jk)[8 * j + 4];
                    a.S[a.s_off[pairs[j]] + 32 * b + lane] = sv;
                    if (a.bmin) {
                        LbConsts k;
                        k.c1 = jk[8 * j + 1];
                        k.c2 = jk[8 * j + 2];
                        k.c3 = jk[8 * j + 3];
                        const float lb = lower_bound(__fmul_rn(__int2float_rn(sv), jk[8 * j]), on, k);
                        const float mn = warp_min(valid ? lb : INFINITY);
                        if (lane == 0) a.bmin[a.s_off[pairs[j]] / 32 + b] = mn;
                    }
                }
            }
        }
        if (!ok) {
            // a copy did not land in time: let this warp's issued copies land,
            // report, and take no further units (the items still run their
            // tables, so every warp keeps to the block's barriers)
            if (lane == 0) {
                us.drain(m);
                if (a.status) atomicOr(a.status, kScanTimeoutBit);
            }
            us.total = 0;
        }
        if (warp == kClaimWarp) claim_item<QB>(a, total, nx, lane);
        __syncthreads();  // tables, jk and the record are reused by the next item
    }
}

}  // namespace erq
