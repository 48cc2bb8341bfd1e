// Query rotation and the coarse (centroid) probe.
//
//   rotate_kernel       Rotator::rotate            inc/index/Rotator.hpp:60-63
//   centroid_dist_kernel L2Sqr16 for every (query, centroid)
//                                                  inc/utils/space.hpp:18-39
//   select_probe_kernel  partial_sort of the nprobe nearest centroids
//                                                  inc/index/Initializer.hpp:55-68
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

// ------------------------------------------------------- probe selection
// One block per query: bitonic sort of (distance, id) keys in shared memory,
// then the nprobe smallest in ascending order.  Also lays out the per-query
// scan workspace: s_off[q][p] = q_slot*stride + sum of 32*blocks(c_p') for
// p' < p, the int32 offset where the scan of (q, p) writes its sums.
__global__ void select_probe_kernel(const float* __restrict__ dist, int nq, int K, int Kpow2,
                                    int nprobe, const uint32_t* __restrict__ c_nblocks,
                                    uint64_t stride, uint32_t* __restrict__ probe_cid,
                                    float* __restrict__ probe_sqy, uint64_t* __restrict__ s_off) {
    extern __shared__ uint64_t keys[];
    const int q = blockIdx.x;
    const float* dq = dist + (size_t)q * K;
    for (int i = threadIdx.x; i < Kpow2; i += blockDim.x)
        keys[i] = i < K ? dist_key(dq[i], (uint32_t)i) : ~0ull;
    __syncthreads();
    for (int size = 2; size <= Kpow2; size <<= 1) {
        for (int stride_ = size >> 1; stride_ > 0; stride_ >>= 1) {
            for (int t = threadIdx.x; t < (Kpow2 >> 1); t += blockDim.x) {
                const int lo = 2 * t - (t & (stride_ - 1));
                const int hi = lo + stride_;
                const bool up = (lo & size) == 0;
                const uint64_t a = keys[lo], b = keys[hi];
                if ((a > b) == up) {
                    keys[lo] = b;
                    keys[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    // outputs + exclusive prefix of 32*nblocks over the probe order (warp 0)
    if (threadIdx.x < 32) {
        uint64_t run = (uint64_t)q * stride;
        for (int p0 = 0; p0 < nprobe; p0 += 32) {
            const int p = p0 + threadIdx.x;
            uint32_t nbv = 0;
            if (p < nprobe) {
                const uint64_t key = keys[p];
                const uint32_t cid = (uint32_t)(key & 0xffffffffu);
                probe_cid[(size_t)q * nprobe + p] = cid;
                probe_sqy[(size_t)q * nprobe + p] = __uint_as_float((uint32_t)(key >> 32));
                nbv = 32u * c_nblocks[cid];
            }
            uint32_t incl = nbv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t n = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)threadIdx.x >= o) incl += n;
            }
            if (p < nprobe) s_off[(size_t)q * nprobe + p] = run + (incl - nbv);
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
}

}  // namespace erq
