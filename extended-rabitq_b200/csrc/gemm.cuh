// Split-BF16 tensor-core GEMM for the two dense contractions of the path:
//   rotation           Q_r = pad(Q) * P               (Rotator::rotate,
//                                                       inc/index/Rotator.hpp:60-63)
//   centroid ranking   <q_r, c> for every centroid     (the inner-product part of
//                                                       L2Sqr16's K distances)
//
// An FP32 operand x is split into bf16 hi = bf16(x) and lo = bf16(x - hi);
// x*y ~ hi_x*hi_y + hi_x*lo_y + lo_x*hi_y (the dropped lo*lo term and the
// split residues are below 2^-15 |x||y|).  The three products are one bf16
// GEMM over a K dimension of 3D: the A rows hold [hi | hi | lo] and the B rows
// [hi | lo | hi], so a single FP32 accumulator sums all three.
//
// GEMM: C[M][N] = A[M][Kd] * B[N][Kd]^T, A and B row-major bf16 (K contiguous),
// FP32 accumulation on mma.sync m16n8k16; 128x128 block tile, 8 warps of
// 64x32, k-step 32, two-stage cp.async pipeline, XOR-swizzled shared tiles
// for conflict-free ldmatrix.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace erq {

// ----------------------------------------------------------------- split
// out[r][0:Cp] , out[r][Cp:2Cp], out[r][2Cp:3Cp] = (hi, hi, lo) when
// a_side, else (hi, lo, hi); columns >= C of `in` read as 0.  Optionally the
// row's squared norm (float32, sequential) into norms[r].
__global__ void split_rows_kernel(const float* __restrict__ in, int R, int C, int Cp,
                                  bool a_side, __nv_bfloat16* __restrict__ out,
                                  float* __restrict__ norms) {
    const int r = blockIdx.x;
    if (r >= R) return;
    const float* src = in + (size_t)r * C;
    __nv_bfloat16* dst = out + (size_t)r * 3 * Cp;
    float nrm = 0.f;
    for (int c = threadIdx.x; c < Cp; c += blockDim.x) {
        const float x = c < C ? src[c] : 0.f;
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
        dst[c] = hi;
        dst[Cp + c] = a_side ? hi : lo;
        dst[2 * Cp + c] = a_side ? lo : hi;
        nrm = fmaf(x, x, nrm);
    }
    if (norms) {
        __shared__ float red[32];
        for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nrm;
        __syncthreads();
        if (threadIdx.x == 0) {
            float s = 0.f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
            norms[r] = s;
        }
    }
}

// ------------------------------------------------------------------ gemm
constexpr int kGemmBM = 128, kGemmBN = 128, kGemmBK = 32;
constexpr int kGemmThreads = 256;

// Epilogue: C = acc, or (ranking) C = rn[row] + cn[col] - 2 * acc, or
// (MLP layers) C = acc + bias[col], then max(C, 0) when relu.
struct GemmEpilogue {
    const float* row_norm = nullptr;
    const float* col_norm = nullptr;
    const float* bias = nullptr;
    bool relu = false;
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                            uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// byte offset of 16-byte chunk `c` (0..3) of tile row `r` (64 bytes per row)
__device__ __forceinline__ uint32_t tile_off(int r, int c) {
    return (uint32_t)(r * 64 + ((c ^ ((r >> 1) & 3)) << 4));
}

__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_tn_kernel(
    const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
    float* __restrict__ Cout, int M, int N, int Kd, GemmEpilogue epi) {
    __shared__ __align__(128) uint8_t smem[2][2][kGemmBM * kGemmBK * 2];  // [stage][A/B]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps, 64 x 32 each
    const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * kGemmBN;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(&smem[0][0][0]);
    constexpr uint32_t kTileBytes = kGemmBM * kGemmBK * 2;

    auto load_stage = [&](int stage, int k0) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int idx = tid + i * kGemmThreads;  // 0..511: row = idx/4, chunk = idx%4
            const int r = idx >> 2, c = idx & 3;
            const int gm = m0 + r, gn = n0 + r;
            const __nv_bfloat16* ga = A + (size_t)min(gm, M - 1) * Kd + k0 + 8 * c;
            const __nv_bfloat16* gb = B + (size_t)min(gn, N - 1) * Kd + k0 + 8 * c;
            const uint32_t so = tile_off(r, c);
            cp_async16(sbase + (stage * 2 + 0) * kTileBytes + so, ga, gm < M);
            cp_async16(sbase + (stage * 2 + 1) * kTileBytes + so, gb, gn < N);
        }
    };

    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

    const int nk = Kd / kGemmBK;
    load_stage(0, 0);
    cp_async_commit();
    for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) load_stage((kt + 1) & 1, (kt + 1) * kGemmBK);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int st = kt & 1;
        const uint32_t sa = sbase + (st * 2 + 0) * kTileBytes;
        const uint32_t sb = sbase + (st * 2 + 1) * kTileBytes;
#pragma unroll
        for (int kk = 0; kk < kGemmBK / 16; ++kk) {
            uint32_t af[4][4], bfr[4][2];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = wm * 64 + i * 16 + (lane & 15);
                const int c = kk * 2 + (lane >> 4);
                ldmatrix_x4(sa + tile_off(r, c), af[i][0], af[i][1], af[i][2], af[i][3]);
            }
#pragma unroll
            for (int j = 0; j < 4; j += 2) {
                const int r = wn * 32 + j * 8 + (lane & 7) + ((lane >> 4) << 3);
                const int c = kk * 2 + ((lane >> 3) & 1);
                ldmatrix_x4(sb + tile_off(r, c), bfr[j][0], bfr[j][1], bfr[j + 1][0], bfr[j + 1][1]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
        }
        __syncthreads();
    }
    // epilogue: accumulator element e of (i, j) is row g (+8 for e >= 2),
    // column 2*(lane%4) + (e&1) of the 16x8 sub-tile
    const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int row = m0 + wm * 64 + i * 16 + g + ((e >> 1) << 3);
                const int col = n0 + wn * 32 + j * 8 + 2 * t4 + (e & 1);
                if (row < M && col < N) {
                    float v = acc[i][j][e];
                    if (epi.row_norm) v = epi.row_norm[row] + epi.col_norm[col] - 2.f * v;
                    if (epi.bias) v += epi.bias[col];
                    if (epi.relu) v = fmaxf(v, 0.f);
                    Cout[(size_t)row * N + col] = v;
                }
            }
}

}  // namespace erq
