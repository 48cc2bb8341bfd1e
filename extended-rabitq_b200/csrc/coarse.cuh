// Query rotation and the coarse (centroid) probe.
//
//   rotate_kernel       Rotator::rotate            inc/index/Rotator.hpp:60-63
//   centroid_dist_kernel L2Sqr16 for every (query, centroid)
//                                                  inc/utils/space.hpp:18-39
// (the nprobe nearest of these exact distances: probe_exact_kernel, probe.cuh)
#pragma once

#include "common.cuh"

namespace erq {

// ----------------------------------------------------------------- rotate
// out[nq][D] = pad(in[nq][DIM] -> D) * P[D][D], FP32 with FMA accumulation.
// 64x64 output tile per 256-thread block, 4x4 outputs per thread, k-step 16.
constexpr int kRotBM = 64, kRotBN = 64, kRotBK = 16;

__global__ void __launch_bounds__(256) rotate_kernel(const float* __restrict__ in, int nq, int DIM,
                                                     const float* __restrict__ P, int D,
                                                     float* __restrict__ out) {
    __shared__ float As[kRotBK][kRotBM + 4];
    __shared__ float Bs[kRotBK][kRotBN + 4];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int row0 = blockIdx.y * kRotBM, col0 = blockIdx.x * kRotBN;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < D; k0 += kRotBK) {
        // A tile: 64 rows x 16 k, transposed into As[k][m]
        for (int i = tid; i < kRotBM * kRotBK; i += 256) {
            const int m = i / kRotBK, kk = i % kRotBK;
            const int r = row0 + m, k = k0 + kk;
            As[kk][m] = (r < nq && k < DIM) ? in[(size_t)r * DIM + k] : 0.f;
        }
        for (int i = tid; i < kRotBK * kRotBN; i += 256) {
            const int kk = i / kRotBN, n = i % kRotBN;
            const int k = k0 + kk, c = col0 + n;
            Bs[kk][n] = (c < D) ? P[(size_t)k * D + c] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kRotBK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = row0 + ty * 4 + i;
        if (r >= nq) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + tx * 4 + j;
            if (c < D) out[(size_t)r * D + c] = acc[i][j];
        }
    }
}

// --------------------------------------------------- centroid distances
// dist[q][c] = L2Sqr16(q, c): lane l of a 16-lane chain accumulates
// fma(t, t, acc) over dims l, l+16, ... in ascending order, then the GCC
// reduce tree.  Tile: 16 queries x 32 centroids per 256-thread block; thread
// (l, cg, qg) owns chain l of queries 4qg..4qg+3 x centroids cg+4j (j<8).
constexpr int kCdTQ = 16, kCdTC = 32, kCdDC = 64, kCdStride = kCdDC + 16;

__global__ void __launch_bounds__(256) centroid_dist_kernel(const float* __restrict__ Q, int nq,
                                                            const float* __restrict__ C, int K,
                                                            int D, float* __restrict__ dist) {
    __shared__ __align__(16) float Qs[kCdTQ][kCdStride];
    __shared__ __align__(16) float Cs[kCdTC][kCdStride];
    const int tid = threadIdx.x;
    const int l = tid & 15, cg = (tid >> 4) & 3, qg = tid >> 6;
    const int q0 = blockIdx.y * kCdTQ, c0 = blockIdx.x * kCdTC;
    float acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    for (int d0 = 0; d0 < D; d0 += kCdDC) {
        // 16x64 + 32x64 floats as float4: 256 + 512 vectors, 3 per thread
        for (int i = tid; i < (kCdTQ + kCdTC) * (kCdDC / 4); i += 256) {
            const int row = i / (kCdDC / 4), c4 = i % (kCdDC / 4);
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (row < kCdTQ) {
                const int q = q0 + row;
                if (q < nq) v = *reinterpret_cast<const float4*>(Q + (size_t)q * D + d0 + 4 * c4);
                *reinterpret_cast<float4*>(&Qs[row][4 * c4]) = v;
            } else {
                const int cc = c0 + row - kCdTQ;
                if (cc < K) v = *reinterpret_cast<const float4*>(C + (size_t)cc * D + d0 + 4 * c4);
                *reinterpret_cast<float4*>(&Cs[row - kCdTQ][4 * c4]) = v;
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kCdDC / 16; ++kk) {
            float qv[4], cv[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) qv[i] = Qs[4 * qg + i][16 * kk + l];
#pragma unroll
            for (int j = 0; j < 8; ++j) cv[j] = Cs[cg + 4 * j][16 * kk + l];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float t = __fsub_rn(qv[i], cv[j]);
                    acc[i][j] = __fmaf_rn(t, t, acc[i][j]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float s = tree16_sum(acc[i][j]);
            const int q = q0 + 4 * qg + i, cc = c0 + cg + 4 * j;
            if (l == 0 && q < nq && cc < K) dist[(size_t)q * K + cc] = s;
        }
}

}  // namespace erq
