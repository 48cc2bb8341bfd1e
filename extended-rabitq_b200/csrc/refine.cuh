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
#include "layout.cuh"

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
    const uint8_t* excode;        // [N][ex_row] device layout (layout.cuh)
    uint64_t ex_row;              // bytes per EX-code row
    const float* xipnorm;         // [N]
    const uint32_t* ids;          // [N]
    const uint32_t* c_first_block; // [K]
    const uint32_t* c_first_vec;   // [K]
    const uint32_t* c_size;        // [K]
    uint32_t* out_ids;            // [nq][k]
    float* out_dists;             // [nq][k] or null
    const int* q_nprobe;          // optional [nq]: clusters probed by each query
    const uint32_t* order;        // optional: block i refines query order[i]
    const float* bmin;            // optional: smallest lower bound per scanned block, at
                                  // s_off/32 + block (blocks above the threshold are skipped)
    unsigned long long* stats;    // optional [4], added to once per query: the reference's
                                  // exact candidates (lower bound below the threshold at
                                  // their block's start), lanes refined (the windows'
                                  // supersets), windows, window blocks
    int nq, D, EX, nprobe, k;
};


// Codes of bytes (lo, lo+1) of w as exact floats: 0x4B0000vv is 2^23 + v.
__device__ __forceinline__ float2 code_pair(uint32_t w, int lo) {
    const float2 big = make_float2(__int_as_float((int)__byte_perm(w, 0x4B000000u, 0x7540u | (uint32_t)lo)),
                                   __int_as_float((int)__byte_perm(w, 0x4B000000u, 0x7540u | (uint32_t)(lo + 1))));
    return fsub2(big, make_float2(8388608.f, 8388608.f));
}

// Codes of step t (0 <= t < 32/SB) of a lane's uint4 as 4 bytes.
template <int SB>
__device__ __forceinline__ uint32_t step_word(const uint4& v, int t) {
    const uint32_t c[4] = {v.x, v.y, v.z, v.w};
    if (SB == 8) return c[t];
    if (SB == 4) return (c[t >> 1] >> (4 * (t & 1))) & 0x0F0F0F0Fu;
    return (c[t >> 2] >> (2 * (t & 3))) & 0x03030303u;
}

// One step of one candidate: accumulators 4r+0..4r+3 of the reference's 16
// (as two pairs) take fma(unit_q[16s + 4r + i], code, acc).
__device__ __forceinline__ void ip_step(float2 acc[2], const float4& u, uint32_t w) {
    acc[0] = ffma2(make_float2(u.x, u.y), code_pair(w, 0), acc[0]);
    acc[1] = ffma2(make_float2(u.z, u.w), code_pair(w, 2), acc[1]);
}

// <unit_q, ex code> of NC (1 or 2) candidates by the 4 lanes r = 0..3 of a
// quad, in the reference's order (IP*_fxu* in inc/utils/space.hpp): the 16
// accumulators acc[l] take the dims l, l+16, l+32, ... in turn; lane r holds
// acc[4r..4r+3].  Rows are in the lane-interleaved layout of layout.cuh;
// each lane streams its own uint4s one ahead (a loop unrolled by 3, then the
// last pass, which fetches nothing).  uq4 = unit_q as float4.
// Returns the sums (the reduce tree: acc[l] + acc[l+8], then + 4, then
// (0 + 2) + (1 + 3)) in every lane of the quad.
template <int SB, int NC>
__device__ __forceinline__ void ex_ip_quad(const float4* __restrict__ uq4, const uint4* __restrict__ row0,
                                           const uint4* __restrict__ row1, int r, int steps,
                                           float out[2]) {
    constexpr int SPU = 32 / SB;  // steps per uint4
    const int U = (steps + SPU - 1) / SPU;
    float2 acc[NC][2];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c][0] = acc[c][1] = make_float2(0.f, 0.f);
    // running pointers: each pass advances them by a constant, so the loads
    // of a pass take immediate offsets
    const uint4* rp[NC];
    rp[0] = row0 + r;
    if (NC > 1) rp[NC - 1] = row1 + r;
    const float4* qp = uq4 + r;
    uint4 cur[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) cur[c] = __ldg(rp[c]);
    const int Uf = steps / SPU;      // uint4s whose steps are all real
    const int Upf = min(Uf, U - 1);  // passes that fetch the next uint4
    int u = 0;
#pragma unroll 3
    for (; u < Upf; ++u) {
        uint4 nn[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            rp[c] += 4;
            nn[c] = __ldg(rp[c]);
        }
#pragma unroll
        for (int t = 0; t < SPU; ++t) {
            const float4 q = qp[4 * t];
#pragma unroll
            for (int c = 0; c < NC; ++c) ip_step(acc[c], q, step_word<SB>(cur[c], t));
        }
        qp += 4 * SPU;
#pragma unroll
        for (int c = 0; c < NC; ++c) cur[c] = nn[c];
    }
    for (; u < Uf; ++u) {  // the last pass: nothing left to fetch
#pragma unroll
        for (int t = 0; t < SPU; ++t) {
            const float4 q = qp[4 * t];
#pragma unroll
            for (int c = 0; c < NC; ++c) ip_step(acc[c], q, step_word<SB>(cur[c], t));
        }
        qp += 4 * SPU;
    }
    for (int t = 0; t < steps - Uf * SPU; ++t) {  // a partly filled last uint4
        const float4 q = qp[4 * t];
#pragma unroll
        for (int c = 0; c < NC; ++c) ip_step(acc[c], q, step_word<SB>(cur[c], t));
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        float t3[4], t6[4];
        const float a4[4] = {acc[c][0].x, acc[c][0].y, acc[c][1].x, acc[c][1].y};
#pragma unroll
        for (int i = 0; i < 4; ++i) t3[i] = __fadd_rn(__shfl_xor_sync(0xffffffffu, a4[i], 2), a4[i]);
#pragma unroll
        for (int i = 0; i < 4; ++i) t6[i] = __fadd_rn(__shfl_xor_sync(0xffffffffu, t3[i], 1), t3[i]);
        out[c] = __fadd_rn(__fadd_rn(t6[0], t6[2]), __fadd_rn(t6[1], t6[3]));
    }
}

constexpr int kRefineThreads = 128;     // 4 warps per query
constexpr int kWindowBlocks = 16;       // blocks whose candidates are refined together
constexpr int kFirstWindowBlocks = 8;   // the same in the query's first probed cluster
// Wide form for small batches (a query per SM): more warps, longer windows.
constexpr int kWideWarps = 32;
constexpr int kWideWindowBlocks = 128;

// Shared memory of one block: unit_q[D] | per window lane: lb, ipq, onorm,
// ex_dist, id, list | pool_d[kpad] | pool_id[kpad] | misc | window blocks
__host__ __device__ constexpr size_t refine_smem_bytes_per_query(int D, int kpad, int wb) {
    return (size_t)D * 4 + (size_t)wb * 32 * (5 * 4 + 2) + (size_t)kpad * 8 + 64 + 128 + (size_t)wb * 4;
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
// scratch.  The caller may drop candidates that cannot enter a full pool
// (distance > its k-th): they would rank >= k and move no other entry.
__device__ __forceinline__ void pool_merge_block(float* pool_d, uint32_t* pool_id, int& size, int k,
                                                 float& distk, bool cand, float d, uint32_t id,
                                                 float* cs, int lane, bool count_all = false) {
    const uint32_t cm = __ballot_sync(0xffffffffu, cand);
    const int nc = __popc(cm);
    // each candidate's place among the pool entries: those below it (a new
    // value goes before equal ones), by binary search on the sorted pool
    const auto place = [&](bool m, float v) {
        int l = 0;
        if (m) {
            int hi = size;
            while (l < hi) {
                const int mid = (l + hi) >> 1;
                if (pool_d[mid] < v) l = mid + 1; else hi = mid;
            }
        }
        return l;
    };
    // Up to kFew candidates (any number with count_all) stay on their lanes:
    // a candidate's rank among the block's candidates is counted by broadcast,
    // and each pool entry counts the candidates below it.  More are sorted
    // (bitonic, lane j then holds the j-th).  Sorting pays while the pool fills
    // (blocks of up to 32 candidates spread over the whole pool); in a query's
    // later clusters counting is cheaper at any number.
    constexpr int kFew = 4;
    const bool few = count_all || nc <= kFew;
    int lo = 0;
    float dv = d;
    uint32_t val = id;
    bool mine = cand;
    int rk = 0;
    if (few) {
        lo = place(cand, d);
        const uint64_t key = merge_key(d, lane, cand);
        for (uint32_t m = cm; m; m &= m - 1u) {
            const int src = __ffs(m) - 1;
            rk += merge_key(__shfl_sync(0xffffffffu, d, src), src, true) < key;
        }
    } else {
        uint64_t key = merge_key(d, lane, cand);
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
        rk = lane;
        mine = lane < nc;
        cs[lane] = dv;
        lo = place(mine, dv);
    }
    // entries below the smallest candidate's place stay put
    const int first = (int)__reduce_min_sync(0xffffffffu, mine ? (uint32_t)lo : 0xffffffffu);
    const int rc = mine ? rk + lo : k;
    __syncwarp();
    // move pool entries, top chunk first: entry i goes to i + c(i) >= i, and
    // i + c(i) strictly increases with i, so no chunk overwrites an entry
    // that has not been read or one already moved
    for (int i0 = ((size - 1) >> 5) << 5; i0 >= 0 && i0 + 31 >= first; i0 -= 32) {
        const int i = i0 + lane;
        float pd = 0.f;
        uint32_t pid = 0u;
        if (i < size) {
            pd = pool_d[i];
            pid = pool_id[i];
        }
        int c = 0;
        if (few) {
            for (uint32_t m = cm; m; m &= m - 1u) c += __shfl_sync(0xffffffffu, d, __ffs(m) - 1) <= pd;
        } else if (i < size) {
            int h2 = nc;
            while (c < h2) {
                const int mid = (c + h2) >> 1;
                if (cs[mid] <= pd) c = mid + 1; else h2 = mid;
            }
        }
        const int pr = i < size ? i + c : k;
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

// One block of WARPS warps per query (4, or 32 in the wide form).  Per window
// of up to WB blocks of the current cluster (16, or 128; 8 in a query's first
// cluster in the 4-warp form): the warps compute the lower bounds of the
// window's blocks, dealt round robin, and list the lanes below the threshold
// as it stands at the window's start (a superset of the exact candidates,
// because the threshold only falls); the quads compute the listed candidates'
// exact distances (8 quads per warp; warps without a candidate skip the
// round); warp 0 then replays the window in the reference's order -
// each block's mask against the threshold at that block's start, the block's
// candidates merged into the pool as inserting them in lane order would.
template <int EX, int WARPS, int WB>
__global__ void __launch_bounds__(WARPS * 32, WARPS == 4 ? 8 : 1) refine_kernel(RefineArgs a) {
    constexpr int kThreads = WARPS * 32, kLanes = WB * 32;
    static_assert(WB % WARPS == 0 && kLanes <= 65536, "window lanes are listed as u16");
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = a.order ? (int)a.order[blockIdx.x] : (int)blockIdx.x;
    const int D = a.D, k = a.k;
    const int kpad = (k + 31) & ~31;
    float* uq = reinterpret_cast<float*>(smem_raw);
    float* w_lb = uq + D;
    float* w_ipq = w_lb + kLanes;
    float* w_on = w_ipq + kLanes;
    float* w_ed = w_on + kLanes;
    uint32_t* w_id = reinterpret_cast<uint32_t*>(w_ed + kLanes);
    uint16_t* w_list = reinterpret_cast<uint16_t*>(w_id + kLanes);
    float* pool_d = reinterpret_cast<float*>(w_list + kLanes);
    uint32_t* pool_id = reinterpret_cast<uint32_t*>(pool_d + kpad);
    int* misc = reinterpret_cast<int*>(pool_id + kpad);  // [0] list count [1] pool size
    float* s_distk = reinterpret_cast<float*>(misc + 2);
    float* cs = reinterpret_cast<float*>(misc + 16);  // 32 floats of merge scratch
    uint32_t* w_blk = reinterpret_cast<uint32_t*>(cs + 32);  // the window's blocks
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
    uint32_t st_cand = 0, st_refined = 0, st_windows = 0, st_blocks = 0;  // with a.stats
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
        const LbConsts lbk = lb_consts(sumq, y, one_over_sqrtD);
        const double ex_sub = __dmul_rn((double)fac_rescale - 0.5, (double)sumq);
        const uint32_t n = a.c_size[cid];
        const uint32_t fb = a.c_first_block[cid];
        const uint32_t first_vec = a.c_first_vec[cid];
        const int32_t* S = a.S + a.s_off[qp];
        const float* bmin = a.bmin ? a.bmin + a.s_off[qp] / 32 : nullptr;
        const uint32_t nblocks = (n + 31) >> 5;
        bool uq_ready = false;
        // The first cluster's threshold falls fast (the pool fills, then
        // tightens), so a long window there lists many lanes that its replay
        // drops; later clusters' thresholds barely move and long windows save
        // barriers.
        const int wcap = (WARPS == 4 && p == 0) ? kFirstWindowBlocks : WB;
        for (uint32_t wb = 0; wb < nblocks;) {
            const float d0 = *s_distk;
            const int filled = misc[1];
            // While the pool is filling every lane is a candidate: take just
            // enough blocks to fill it, so few lanes are refined in vain.
            const int want = filled < k ? min(wcap, max(1, (k - filled + 31) / 32))
                                        : wcap;
            __syncthreads();
            // warp 0 picks the window: the next `want` blocks from wb whose
            // smallest lower bound is below the threshold (a block above it
            // has no candidate now or later: the threshold only falls)
            if (warp == 0) {
                int got = 0;
                uint32_t pos = wb, next = nblocks;
                while (got < want && pos < nblocks) {
                    const uint32_t bb = pos + lane;
                    const bool take = bb < nblocks && (!bmin || bmin[bb] < d0);
                    const uint32_t m = __ballot_sync(0xffffffffu, take);
                    const int rank = __popc(m & ((1u << lane) - 1u));
                    if (take && got + rank < want) w_blk[got + rank] = bb;
                    const int nm = __popc(m);
                    if (got + nm >= want) {
                        // the want-th taken block ends the window
                        const uint32_t endm = __ballot_sync(0xffffffffu, take && rank == want - got - 1);
                        next = pos + (uint32_t)(__ffs(endm) - 1) + 1;
                        got = want;
                        break;
                    }
                    got += nm;
                    pos += 32;
                }
                if (lane == 0) {
                    misc[0] = 0;
                    misc[5] = got;
                    misc[6] = (int)next;
                }
            }
            __syncthreads();
            const int nbw = misc[5];
            const uint32_t wnext = (uint32_t)misc[6];
            // lower bounds and the candidate superset, 4 blocks per warp
#pragma unroll
            for (int i = 0; i < WB / (kThreads / 32); ++i) {
                const int b = i * (kThreads / 32) + warp;  // round robin: short windows use every warp
                if (b < nbw) {  // uniform per warp
                    const uint32_t blk = w_blk[b];
                    const float ipq = __fmul_rn(__int2float_rn(S[32 * blk + lane]), delta);
                    const float on = a.onorm[(size_t)(fb + blk) * 32 + lane];
                    const float t = lower_bound(ipq, on, lbk);
                    const bool valid = 32 * blk + lane < n;
                    // padding lanes never pass (NaN compares false)
                    w_lb[32 * b + lane] = valid ? t : __int_as_float(0x7fc00000);
                    w_ipq[32 * b + lane] = ipq;
                    w_on[32 * b + lane] = on;
                    const uint32_t m = __ballot_sync(0xffffffffu, valid && t < d0);
                    int base = 0;
                    if (lane == 0 && m) base = atomicAdd(&misc[0], __popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if ((m >> lane) & 1u) {
                        w_list[base + __popc(m & ((1u << lane) - 1u))] = (uint16_t)(32 * b + lane);
                        // start the candidate's EX-code row on its way to L2
                        const size_t pos = (size_t)first_vec + 32 * blk + lane;
                        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                                         a.excode + pos * a.ex_row),
                                     "r"((uint32_t)a.ex_row)
                                     : "memory");
                    }
                }
            }
            __syncthreads();
            const int cnt = misc[0];
            if (a.stats) {
                st_refined += cnt;
                st_windows += 1;
                st_blocks += nbw;
            }
            if (cnt == 0) {  // uniform: nothing in this window can pass
                wb = wnext;
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
            // refine the listed candidates: quad g (lanes 4g..4g+3) takes two
            // per round while more than one per quad remain, else one; within a warp
            // that has work, quads past the end repeat the list's first so
            // the warp stays converged
            {
                const int g = tid >> 2, r = tid & 3;
                const float4* uq4 = reinterpret_cast<const float4*>(uq);
                for (int base = 0; base < cnt;) {
                    const int two = cnt - base > kThreads / 4;
                    const int step = two ? kThreads / 2 : kThreads / 4;
                    // per warp: skip when none of its slots holds a candidate,
                    // one candidate per quad when its second slots are empty
                    if (base + 8 * warp >= cnt) {
                        base += step;
                        continue;
                    }
                    const int wtwo = two && base + kThreads / 4 + 8 * warp < cnt;
                    const int i0 = base + g, i1 = base + kThreads / 4 + g;
                    const int s0 = w_list[i0 < cnt ? i0 : 0];
                    const int s1 = w_list[wtwo && i1 < cnt ? i1 : 0];
                    const size_t pos0 = (size_t)first_vec + 32 * w_blk[s0 >> 5] + (s0 & 31);
                    const size_t pos1 = (size_t)first_vec + 32 * w_blk[s1 >> 5] + (s1 & 31);
                    const uint4* row0 = reinterpret_cast<const uint4*>(a.excode + pos0 * a.ex_row);
                    const uint4* row1 = reinterpret_cast<const uint4*>(a.excode + pos1 * a.ex_row);
                    // lane 0 of the quad finishes the first, lane 1 the second
                    const int i = r == 0 ? i0 : i1;
                    const bool fin = r < 2 && (r == 0 || wtwo) && i < cnt;
                    const int slot = r == 0 ? s0 : s1;
                    const size_t pos = r == 0 ? pos0 : pos1;
                    float xipn = 0.f;
                    uint32_t vid = 0u;
                    if (fin) {
                        xipn = __ldg(a.xipnorm + pos);
                        vid = __ldg(a.ids + pos);
                    }
                    float ip[2];
                    if (wtwo)
                        ex_ip_quad<ex_storage_bits(EX), 2>(uq4, row0, row1, r, D / 16, ip);
                    else
                        ex_ip_quad<ex_storage_bits(EX), 1>(uq4, row0, row0, r, D / 16, ip);
                    if (fin) {
                        // inc/index/HASearcher.hpp:225-232
                        const float on = w_on[slot];
                        const float sqr_x = __fmul_rn(on, on);
                        const float t = __fadd_rn(__fmul_rn((float)fac_rescale, w_ipq[slot]), r == 0 ? ip[0] : ip[1]);
                        const double br = __dsub_rn((double)t, ex_sub);
                        const float xy = __fmul_rn(xipn, y);
                        const float f = __fadd_rn(sqr_x, sqy);
                        w_ed[slot] = __double2float_rn(__dsub_rn((double)f, __dmul_rn((double)xy, br)));
                        w_id[slot] = vid;
                    }
                    base += step;
                }
            }
            __syncthreads();
            if (warp == 0) {
                for (int b = 0; b < nbw; ++b) {
                    // candidates of the block against the threshold at its
                    // start; those above a full pool's k-th cannot enter
                    const float ed = w_ed[32 * b + lane];
                    const bool below = w_lb[32 * b + lane] < distk;
                    if (a.stats) st_cand += __popc(__ballot_sync(0xffffffffu, below));
                    const bool enter = below && (size < k || !(ed > distk));
                    if (__ballot_sync(0xffffffffu, enter))
                        pool_merge_block(pool_d, pool_id, size, k, distk, enter, ed,
                                         w_id[32 * b + lane], cs, lane, p > 0);
                }
                if (lane == 0) {
                    *s_distk = distk;
                    misc[1] = size;
                }
            }
            __syncthreads();
            wb = wnext;
        }
    }
    if (warp == 0) {
        if (a.stats && lane == 0) {
            atomicAdd(a.stats + 0, (unsigned long long)st_cand);
            atomicAdd(a.stats + 1, (unsigned long long)st_refined);
            atomicAdd(a.stats + 2, (unsigned long long)st_windows);
            atomicAdd(a.stats + 3, (unsigned long long)st_blocks);
        }
        uint32_t* oid = a.out_ids + (size_t)q * k;
        for (int i = lane; i < k; i += 32) {
            oid[i] = i < size ? pool_id[i] : 0u;
            if (a.out_dists)
                a.out_dists[(size_t)q * k + i] = i < size ? pool_d[i] : __int_as_float(0x7f800000);
        }
    }
}

}  // namespace erq
