// Lloyd k-means for the IVF clustering step.
//
// The reference clusters its data with faiss (python/ivf.py:5-34:
// index_factory("IVF{K},Flat").train, i.e. faiss::Clustering 1.8.0): initial
// centroids are K distinct data points drawn at random, then each iteration
// assigns every point to its nearest centroid, moves each centroid to the
// mean of its points, and re-seeds every empty cluster by splitting a
// populated one (the two centroids become c * (1 +- eps) alternately per
// dimension, eps = 1/1024, and the points are shared).
//
// Here one iteration is
//   1. distance ranks ||x||^2 + ||c||^2 - 2 x.c on the tensor cores (the
//      split-BF16 GEMM of gemm_tc.cuh, about FP32 accuracy), in row chunks;
//   2. argmin_rows_kernel: the nearest centroid of each point (ties: the
//      smaller index);
//   3. kmeans_accumulate_kernel: per-cluster sums in 64-bit fixed point
//      (scale 2^s, s <= 32 chosen so that n * max|x| * 2^s < 2^62), so the
//      integer atomics give the same sums in any order and the clustering is
//      deterministic;
//   4. kmeans_update_kernel: means in double, rounded to float;
//   5. empty clusters split on the host's choice (splitmix64 stream).
#pragma once

#include <cstdint>

#include "common.cuh"

namespace erq {

// One warp per row of dist [rows][K]: the column of the smallest value
// (smallest index among equal ones).
__global__ void argmin_rows_kernel(const float* __restrict__ dist, int rows, int K,
                                   uint32_t* __restrict__ assign) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= rows) return;
    const float* r = dist + (size_t)warp * K;
    float best = INFINITY;
    int bi = 0x7fffffff;
    for (int c = lane; c < K; c += 32) {
        const float v = r[c];
        if (v < best) {  // ascending c per lane: the first minimum stays
            best = v;
            bi = c;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov < best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
        }
    }
    if (lane == 0) assign[warp] = (uint32_t)(bi == 0x7fffffff ? 0 : bi);
}

// sums[c][d] += round(x[i][d] * scale), counts[c] += 1 for c = assign[i].
// One block per 8 points, a thread per (point, dim) column stripe.
__global__ void kmeans_accumulate_kernel(const float* __restrict__ x, int n, int dim,
                                         double scale, const uint32_t* __restrict__ assign,
                                         unsigned long long* __restrict__ sums,
                                         uint32_t* __restrict__ counts) {
    const int i0 = blockIdx.x * 8;
    for (int p = 0; p < 8; ++p) {
        const int i = i0 + p;
        if (i >= n) return;
        const uint32_t c = assign[i];
        if (threadIdx.x == 0) atomicAdd(counts + c, 1u);
        const float* xi = x + (size_t)i * dim;
        unsigned long long* sc = sums + (size_t)c * dim;
        for (int d = threadIdx.x; d < dim; d += blockDim.x)
            atomicAdd(sc + d, (unsigned long long)__double2ll_rn((double)xi[d] * scale));
    }
}

// cent[c] = sums[c] / counts[c] for populated clusters (others keep theirs).
__global__ void kmeans_update_kernel(const unsigned long long* __restrict__ sums,
                                     const uint32_t* __restrict__ counts, int K, int dim,
                                     double scale, float* __restrict__ cent) {
    const size_t n = (size_t)K * dim;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const uint32_t cnt = counts[t / dim];
        if (cnt == 0) continue;
        const double s = (double)(long long)sums[t] / scale;
        cent[t] = (float)(s / (double)cnt);
    }
}

// Empty cluster ci re-seeded from cj: c_ci = c_cj * (1 + eps s_d),
// c_cj = c_cj * (1 - eps s_d), s_d = +1 on even dims, -1 on odd ones.
__global__ void kmeans_split_kernel(float* __restrict__ cent, int dim, int ci, int cj, float eps) {
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < dim; d += gridDim.x * blockDim.x) {
        const float s = (d & 1) ? -eps : eps;
        const float v = cent[(size_t)cj * dim + d];
        cent[(size_t)ci * dim + d] = v * (1.f + s);
        cent[(size_t)cj * dim + d] = v * (1.f - s);
    }
}

// Largest |x| over n values (as float bits: non-negative floats order as
// their bits), into *out (zeroed before).
__global__ void abs_max_kernel(const float* __restrict__ x, size_t n, unsigned* __restrict__ out) {
    float m = 0.f;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[t]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// out[j] = x[rows[j]]
__global__ void gather_rows_kernel(const float* __restrict__ x, int dim, const uint64_t* __restrict__ rows,
                                   int k, float* __restrict__ out) {
    const size_t n = (size_t)k * dim;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t j = t / dim;
        out[t] = x[rows[j] * dim + (t - j * dim)];
    }
}

}  // namespace erq
