// C = A * B^T on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// A [M][Kd] and B [N][Kd] are BF16, K-major (the split-BF16 operands of
// gemm.cuh: [hi | hi | lo] x [hi | lo | hi] gives hi.hi + hi.lo + lo.hi), the
// accumulators are FP32 in tensor memory.  The kernel is persistent: one CTA
// per SM walks the 128 x 256 output tiles (row-major tile order, so the CTAs
// running at the same time share A tiles in L2), and the shared ring runs on
// across tiles:
//   warp 0   (one thread)  TMA: 64-wide K slices of A (128 rows) and B (256
//            rows), 128-byte swizzled, into a kTcStages-deep shared ring;
//   warp 1   (one thread)  allocates 2 x 256 TMEM columns (two accumulators),
//            issues tcgen05.mma.cta_group::1.kind::f16 (M 128, N 256, K 16)
//            four times per slice into the accumulator of the tile, frees
//            each slot with tcgen05.commit, and commits the accumulator;
//   warps 2-5              read an accumulator back (tcgen05.ld 32x32b, each
//            warp the 32 TMEM lanes of its quadrant), release it, and apply
//            the epilogue of gemm.cuh (plain, distance ranking, bias + ReLU)
//            while the MMAs of the next tile fill the other accumulator.
// Barriers: full/empty per ring slot, tfull/tempty per accumulator, and a
// drain barrier the MMA thread commits to last.  Every mbarrier wait is
// bounded; a wait that runs out sets bit 0 of *status, and the CTA stops
// issuing work, lets its TMA copies land and its MMAs finish, frees its TMEM
// and exits.  Every TMA load reads this GPU's own memory into this CTA's own
// shared memory.
#pragma once

#include <cuda.h>

#include "gemm.cuh"
#include "mbarrier.cuh"

namespace erq {

constexpr int kTcBM = 128, kTcBN = 256, kTcBK = 64, kTcStages = 4;
constexpr int kTcThreads = 192;
constexpr uint32_t kTcABytes = kTcBM * kTcBK * 2;   // 16 KB
constexpr uint32_t kTcBBytes = kTcBN * kTcBK * 2;   // 32 KB
constexpr uint32_t kTcStageBytes = kTcABytes + kTcBBytes;
constexpr uint32_t kTcWaitLimit = 1u << 26;  // polls per pipeline wait (the default)


__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, rows of 128
// bytes, 8-row groups 1024 bytes apart (leading offset unused: 1).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
           (2ull << 61);
}

// Instruction descriptor: F32 accumulator, BF16 A and B, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

constexpr int kTpAccumCols = 256;  // columns per accumulator (two of them)

// 1024 bytes of alignment slack + the ring + barriers and the TMEM address
__host__ __device__ constexpr size_t gemm_tc_smem_bytes() {
    return 1024 + (size_t)kTcStages * kTcStageBytes + 256;
}

__device__ __forceinline__ void gemm_epilogue_store(const uint32_t (&v)[32], float* __restrict__ Cout,
                                                    int M, int N, int row, int col0,
                                                    const GemmEpilogue& epi) {
    if (row >= M) return;
    float* out = Cout + (size_t)row * N;
    const float rn = epi.row_norm ? epi.row_norm[row] : 0.f;
#pragma unroll
    for (int j = 0; j < 32; j += 4) {
        const int col = col0 + j;
        float x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int cc = min(col + e, N - 1);
            x[e] = __uint_as_float(v[j + e]);
            if (epi.row_norm) x[e] = rn + epi.col_norm[cc] - 2.f * x[e];
            if (epi.bias) x[e] += epi.bias[cc];
            if (epi.relu) x[e] = fmaxf(x[e], 0.f);
        }
        if (col + 3 < N && (N & 3) == 0) {
            *reinterpret_cast<float4*>(out + col) = make_float4(x[0], x[1], x[2], x[3]);
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (col + e < N) out[col + e] = x[e];
        }
    }
}

__global__ void __launch_bounds__(kTcThreads, 1) gemm_tc_kernel(
    const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b,
    float* __restrict__ Cout, int M, int N, int Kd, GemmEpilogue epi, uint32_t* status,
    uint32_t wait_limit) {
    extern __shared__ uint8_t smem_raw[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t ring = (raw + 1023u) & ~1023u;
    const uint32_t bars = ring + kTcStages * kTcStageBytes;
    const uint32_t full0 = bars, empty0 = bars + 8 * kTcStages;
    const uint32_t tfull0 = bars + 16 * kTcStages, tempty0 = tfull0 + 16, drain = tempty0 + 16;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_raw + (drain + 8 - raw));
    volatile uint32_t* flag = tmem_slot + 1;  // set when any wait of this CTA ran out
    const int tiles_n = (N + kTcBN - 1) / kTcBN;
    const int tiles = ((M + kTcBM - 1) / kTcBM) * tiles_n;
    const int nk = Kd / kTcBK;

    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(tfull0 + 8 * b, 1);
            mbar_init(tempty0 + 8 * b, 4);  // one arrival per epilogue warp
        }
        mbar_init(drain, 1);
        *flag = 0u;
        mbar_init_fence();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                     "r"((uint32_t)(2 * kTpAccumCols))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    uint32_t issued = 0;  // ring slices the TMA thread started
    if (warp == 0) {
        if (lane == 0) {
            for (int t = blockIdx.x; t < tiles && !*flag; t += gridDim.x) {
                const int m0 = (t / tiles_n) * kTcBM, n0 = (t % tiles_n) * kTcBN;
                for (int kt = 0; kt < nk; ++kt) {
                    const uint32_t s = issued % kTcStages, r = issued / kTcStages;
                    if (r > 0 && !mbar_wait(empty0 + 8 * s, (r - 1) & 1u, wait_limit)) {
                        *flag = 1u;
                        break;
                    }
                    if (*flag) break;
                    const uint32_t sa = ring + s * kTcStageBytes, sb = sa + kTcABytes;
                    mbar_expect_tx(full0 + 8 * s, kTcStageBytes);
                    tma_load_2d(sa, &tma_a, kt * kTcBK, m0, full0 + 8 * s);
                    tma_load_2d(sb, &tma_b, kt * kTcBK, n0, full0 + 8 * s);
                    ++issued;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_bf16(kTcBM, kTcBN);
            uint32_t g = 0;  // ring slices consumed
            int i = 0;       // tiles of this CTA
            for (int t = blockIdx.x; t < tiles && !*flag; t += gridDim.x, ++i) {
                const int b = i & 1;
                const uint32_t u = (uint32_t)(i >> 1);
                if (u > 0 && !mbar_wait(tempty0 + 8 * b, (u - 1) & 1u, wait_limit)) {
                    *flag = 1u;
                    break;
                }
                tc_fence_after();
                const uint32_t acc_tmem = tmem + (uint32_t)(b * kTpAccumCols);
                bool ok = true;
                for (int kt = 0; kt < nk; ++kt, ++g) {
                    const uint32_t s = g % kTcStages, r = g / kTcStages;
                    if (!mbar_wait(full0 + 8 * s, r & 1u, wait_limit) || *flag) {
                        *flag = 1u;
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = ring + s * kTcStageBytes, sb = sa + kTcABytes;
#pragma unroll
                    for (int kk = 0; kk < kTcBK / 16; ++kk) {
                        const uint64_t ad = umma_desc_sw128(sa + 32 * kk);
                        const uint64_t bd = umma_desc_sw128(sb + 32 * kk);
                        const uint32_t acc = (kt | kk) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                            ::"r"(acc_tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                 ::"r"(empty0 + 8 * s)
                                 : "memory");
                }
                if (!ok) break;
                // the accumulator is complete once every MMA above has finished
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(tfull0 + 8 * b)
                             : "memory");
            }
            // every MMA this thread issued has finished once this arrives
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(drain)
                         : "memory");
            mbar_wait(drain, 0, kTcWaitLimit);
        }
    } else {
        const int q = warp & 3;  // TMEM lane quadrant this warp may read
        int i = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++i) {
            const int b = i & 1;
            const uint32_t u = (uint32_t)(i >> 1);
            if (!mbar_wait(tfull0 + 8 * b, u & 1u, wait_limit) || *flag) {
                *flag = 1u;
                break;
            }
            tc_fence_after();
            const int m0 = (t / tiles_n) * kTcBM, n0 = (t % tiles_n) * kTcBN;
            const int row = m0 + 32 * q + lane;
            for (int c0 = 0; c0 < kTcBN; c0 += 32) {
                uint32_t v[32];
                const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * kTpAccumCols + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                      "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
                      "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
                      "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
                      "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (c0 + kTcBN / 8 >= kTcBN) {
                    // the last columns are in registers: the accumulator is free
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(tempty0 + 8 * b);
                }
                gemm_epilogue_store(v, Cout, M, N, row, n0 + c0, epi);
            }
        }
    }
    // A CTA that gave up still lets its TMA copies land before it exits (its
    // MMAs finished above: the MMA thread always waits for the drain commit).
    if (warp == 0 && lane == 0 && *flag) {
        for (uint32_t g = issued > (uint32_t)kTcStages ? issued - kTcStages : 0u; g < issued; ++g)
            mbar_wait(full0 + 8 * (g % kTcStages), (g / kTcStages) & 1u, kTcWaitLimit);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"((uint32_t)(2 * kTpAccumCols))
                     : "memory");
    }
    if (tid == 0 && *flag && status) atomicOr(status, 1u);
}

}  // namespace erq
