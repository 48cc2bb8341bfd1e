// Index construction on the GPU: IVF::construct (inc/index/IVF.hpp:116-153)
// with DataQuantizer::quantize (inc/index/Quantizer.hpp:233-311) for every
// cluster, HIGH_ACC_FAST_SCAN format, writing the bytes the reference's
// create_index writes for the same data, centroids, cluster ids and rotation.
//
// Vectors are processed in file order: clusters in order, each cluster's
// members by ascending data index (IVF::construct's IDLists).  Per vector:
//   build_rotate_kernel   XP = pad(x) P - pad(c) P, every product summed in
//                         ascending k with separate multiply and add
//                         (data_transformation, Quantizer.hpp:316-362, whose
//                         matrix product accumulates that way)
//   build_rows_kernel     ||XP|| in double (ascending dims), XP / ||XP|| in
//                         float, the sign bits (XP > 0)
//   build_x2_kernel       L2Sqr(x, c) over DIM (16 FMA chains + the reduce
//                         tree, then the tail in order) and ||o - c|| =
//                         sqrt((double) that) (rabitq_factor, Quantizer.hpp:386-437)
//   fast_quantize_kernel  the EX-bit code: fast_quantize's sweep over the
//                         critical rescaling factors (Quantizer.hpp:138-219),
//                         one thread per vector with its priority queue of
//                         (t, dim) in global memory, every double step as the
//                         reference takes it
//   build_long_kernel     codes flipped on negative dims, store_compacted_code
//                         (Quantizer.hpp:491-631), xipnorm = ipnorm * 2 * ||o - c||
//   build_short_kernel    the 1-bit FastScan blocks (pack_binary + pack_codes,
//                         Quantizer.hpp:371-384, fastscan/pack_codes.hpp:33-98)
//                         and the block factor ||o - c||; lanes past the
//                         cluster's end hold zero codes and factor 0 (the
//                         reference leaves those factors unset)
#pragma once

#include <cstdint>

#include "common.cuh"

namespace erq {

constexpr int kBuildBM = 64, kBuildBN = 64, kBuildBK = 16;

// out[r][j] = sum_{k < D} xp[r][k] P[k][j] (ascending k, multiply then add),
// xp = row order[r] of x padded with zeros from DIM to D; minus sub[cid[r]][j]
// when sub is given.  64 x 64 output tile per 256-thread block, 4 x 4 per
// thread.
__global__ void __launch_bounds__(256) build_rotate_kernel(const float* __restrict__ x, int DIM,
                                                           const uint32_t* __restrict__ order, int n,
                                                           const float* __restrict__ P, int D,
                                                           const float* __restrict__ sub,
                                                           const uint32_t* __restrict__ cid,
                                                           float* __restrict__ out) {
    __shared__ float As[kBuildBK][kBuildBM + 4];
    __shared__ float Bs[kBuildBK][kBuildBN + 4];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int row0 = blockIdx.y * kBuildBM, col0 = blockIdx.x * kBuildBN;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    for (int k0 = 0; k0 < D; k0 += kBuildBK) {
        for (int i = tid; i < kBuildBM * kBuildBK; i += 256) {
            const int m = i / kBuildBK, kk = i % kBuildBK;
            const int r = row0 + m, k = k0 + kk;
            float v = 0.f;
            if (r < n && k < DIM) v = x[(size_t)(order ? order[r] : (uint32_t)r) * DIM + k];
            As[kk][m] = v;
        }
        for (int i = tid; i < kBuildBK * kBuildBN; i += 256) {
            const int kk = i / kBuildBN, c = i % kBuildBN;
            Bs[kk][c] = (col0 + c < D) ? P[(size_t)(k0 + kk) * D + col0 + c] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBuildBK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(a[i], b[j]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = row0 + ty * 4 + i;
        if (r >= n) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + tx * 4 + j;
            if (c >= D) continue;
            float v = acc[i][j];
            if (sub) v = __fsub_rn(v, sub[(size_t)cid[r] * D + c]);
            out[(size_t)r * D + c] = v;
        }
    }
}

// One thread per row of xp [n][D]: sq = sum of double(x)^2 in ascending
// dims, norm = (float)sqrt(sq); xp becomes x / norm (unchanged when sq = 0,
// rowwise().normalized()); bits[r][w] bit i = (x_{64w+i} > 0).
__global__ void build_rows_kernel(float* __restrict__ xp, int n, int D, uint64_t* __restrict__ bits) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    float* row = xp + (size_t)r * D;
    double sq = 0.0;
    for (int j = 0; j < D; ++j) {
        const double v = (double)row[j];
        sq = __dadd_rn(sq, __dmul_rn(v, v));
    }
    const float norm = __double2float_rn(__dsqrt_rn(sq));
    for (int w = 0; w < D / 64; ++w) {
        uint64_t b = 0;
        for (int i = 0; i < 64; ++i) {
            const float v = row[64 * w + i];
            b |= (uint64_t)(v > 0.f) << i;
            if (sq > 0.0) row[64 * w + i] = __fdiv_rn(v, norm);
        }
        bits[(size_t)r * (D / 64) + w] = b;
    }
}

// ||o - c|| of each row: L2Sqr (inc/utils/space.hpp:18-51) over DIM of the
// raw vector and its raw centroid, then sqrt in double rounded to float.
// One half-warp per row.
__global__ void build_x2_kernel(const float* __restrict__ x, const uint32_t* __restrict__ order,
                                const float* __restrict__ cent, const uint32_t* __restrict__ cid,
                                int n, int DIM, float* __restrict__ onorm) {
    const int hw = (blockIdx.x * blockDim.x + threadIdx.x) >> 4, l = threadIdx.x & 15;
    const int r = min(hw, n - 1);
    const float* a = x + (size_t)order[r] * DIM;
    const float* c = cent + (size_t)cid[r] * DIM;
    const int num16 = DIM - (DIM & 15);
    float acc = 0.f;
    for (int i = l; i < num16; i += 16) {
        const float t = __fsub_rn(a[i], c[i]);
        acc = __fmaf_rn(t, t, acc);
    }
    float s = tree16_sum(acc);
    if (l == 0 && hw < n) {
        for (int i = num16; i < DIM; ++i) {
            const float t = __fsub_rn(a[i], c[i]);
            s = __fadd_rn(s, __fmul_rn(t, t));
        }
        onorm[hw] = __double2float_rn(__dsqrt_rn((double)s));
    }
}

// fast_quantize (inc/index/Quantizer.hpp:138-219) for rows [row0, row0 + T)
// of xn, one thread per row.  The thread's priority queue of (t, dim),
// ordered by t then dim as std::priority_queue<pair, ..., greater> pops them,
// and its current codes live in global memory, entry e of thread j at
// e * T + j.  code[r][i] = the EX-bit magnitude code of |xn[r][i]|,
// ipnorm[r] = 1 / sum (code + 0.5) |xn| (1 when not finite).
__global__ void fast_quantize_kernel(const float* __restrict__ xn, int rows, int row0, int T, int D,
                                     int EX, double* __restrict__ heap_t,
                                     uint16_t* __restrict__ heap_i, uint8_t* __restrict__ cur,
                                     uint8_t* __restrict__ code, float* __restrict__ ipnorm) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = row0 + j;
    if (j >= T || r >= rows) return;
    const float* o = xn + (size_t)r * D;
    const double eps = 1e-5;
    const int cap = (1 << EX) - 1;
    double max_o = -1.0;
    for (int i = 0; i < D; ++i) {
        const double v = (double)fabsf(o[i]);
        if (v > max_o) max_o = v;
    }
    const double t_start = __ddiv_rn((double)(cap / 3), max_o);
    const double t_end = __ddiv_rn((double)(cap + 10), max_o);
    double sqr_den = (double)D * 0.25;
    double num = 0.0;
    auto ht = [&](int e) -> double& { return heap_t[(size_t)e * T + j]; };
    auto hi = [&](int e) -> uint16_t& { return heap_i[(size_t)e * T + j]; };
    auto less = [](double ta, int ia, double tb, int ib) { return ta < tb || (ta == tb && ia < ib); };
    for (int i = 0; i < D; ++i) {
        const double v = (double)fabsf(o[i]);
        const int c = __double2int_rz(__dadd_rn(__dmul_rn(t_start, v), eps));
        cur[(size_t)i * T + j] = (uint8_t)c;
        sqr_den = __dadd_rn(sqr_den, (double)(c * c + c));
        num = __dadd_rn(num, __dmul_rn((double)c + 0.5, v));
        ht(i) = __ddiv_rn((double)(c + 1), v);
        hi(i) = (uint16_t)i;
    }
    // heapify (the pop order of distinct keys does not depend on the layout)
    int size = D;
    auto sift = [&](int e) {
        const double t0 = ht(e);
        const int i0 = hi(e);
        while (true) {
            const int a = 2 * e + 1;
            if (a >= size) break;
            int m = a;
            double tm = ht(a);
            int im = hi(a);
            if (a + 1 < size) {
                const double tb = ht(a + 1);
                const int ib = hi(a + 1);
                if (less(tb, ib, tm, im)) {
                    m = a + 1;
                    tm = tb;
                    im = ib;
                }
            }
            if (!less(tm, im, t0, i0)) break;
            ht(e) = tm;
            hi(e) = (uint16_t)im;
            e = m;
        }
        ht(e) = t0;
        hi(e) = (uint16_t)i0;
    };
    for (int e = size / 2 - 1; e >= 0; --e) sift(e);
    double max_ip = 0.0, t = 0.0;
    while (size > 0) {
        const double cur_t = ht(0);
        const int id = hi(0);
        const int c = (int)cur[(size_t)id * T + j] + 1;
        cur[(size_t)id * T + j] = (uint8_t)c;
        const double v = (double)fabsf(o[id]);
        sqr_den = __dadd_rn(sqr_den, (double)(2 * c));
        num = __dadd_rn(num, v);
        const double ip = __ddiv_rn(num, __dsqrt_rn(sqr_den));
        if (ip > max_ip) {
            max_ip = ip;
            t = cur_t;
        }
        bool again = false;
        double tn = 0.0;
        if (c < cap) {
            tn = __ddiv_rn((double)(c + 1), v);
            again = tn < t_end;
        }
        if (again) {  // pop then push = the new entry at the root, sifted down
            ht(0) = tn;
            hi(0) = (uint16_t)id;
        } else {
            --size;
            if (size == 0) break;
            ht(0) = ht(size);
            hi(0) = hi(size);
        }
        sift(0);
    }
    double num2 = 0.0;
    uint8_t* out = code + (size_t)r * D;
    for (int i = 0; i < D; ++i) {
        const double v = (double)fabsf(o[i]);
        int b = __double2int_rz(__dadd_rn(__dmul_rn(t, v), eps));
        if (b >= (1 << EX)) b = cap;
        num2 = __dadd_rn(num2, __dmul_rn((double)b + 0.5, v));
        out[i] = (uint8_t)b;
    }
    float ipn = __double2float_rn(__ddiv_rn(1.0, num2));
    if (!isfinite(ipn)) ipn = 1.f;
    ipnorm[r] = ipn;
}

// Per row: codes flipped where the sign bit is 0, compacted to D*EX/8 bytes
// (store_compacted_code), xipnorm = (ipnorm * 2) * onorm.  One thread per
// (row, 64-dim group).
__global__ void build_long_kernel(const uint8_t* __restrict__ code, const uint64_t* __restrict__ bits,
                                  const float* __restrict__ ipnorm, const float* __restrict__ onorm,
                                  int rows, int D, int EX, uint8_t* __restrict__ lng,
                                  float* __restrict__ xipnorm) {
    const int G = D / 64;
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= (size_t)rows * G) return;
    const int r = (int)(t / G), g = (int)(t - (size_t)r * G);
    const uint8_t mask = (uint8_t)((1 << EX) - 1);
    const uint64_t sb = bits[(size_t)r * G + g];
    uint8_t v[64];
    for (int i = 0; i < 64; ++i) {
        const uint8_t c = code[(size_t)r * D + 64 * g + i];
        v[i] = ((sb >> i) & 1) ? c : (uint8_t)(~c & mask);
    }
    const size_t row_bytes = (size_t)D * EX / 8;
    uint8_t* o = lng + (size_t)r * row_bytes + (size_t)g * 8 * EX;
    if (EX == 8) {
        for (int i = 0; i < 64; ++i) o[i] = v[i];
    } else if (EX == 4) {
        for (int h = 0; h < 2; ++h)
            for (int i = 0; i < 16; ++i) o[16 * h + i] = v[32 * h + i] | (uint8_t)(v[32 * h + 16 + i] << 4);
    } else if (EX == 2 || EX == 3) {
        for (int i = 0; i < 16; ++i)
            o[i] = (v[i] & 3) | ((v[16 + i] & 3) << 2) | ((v[32 + i] & 3) << 4) | ((v[48 + i] & 3) << 6);
        if (EX == 3)  // top byte m, bit j = bit 2 of dim 8j + m
            for (int m = 0; m < 8; ++m) {
                uint8_t b = 0;
                for (int jj = 0; jj < 8; ++jj) b |= (uint8_t)(((v[8 * jj + m] >> 2) & 1) << jj);
                o[16 + m] = b;
            }
    } else {  // 6 or 7
        const uint8_t lo = EX == 7 ? 0x3F : 0xFF;
        for (int i = 0; i < 16; ++i) {
            o[i] = (v[i] & lo) | (uint8_t)((v[32 + i] << 2) & 0xC0);
            o[16 + i] = (v[16 + i] & lo) | (uint8_t)((v[48 + i] << 2) & 0xC0);
            o[32 + i] = (v[32 + i] & 0x0F) | (uint8_t)((v[48 + i] & 0x0F) << 4);
        }
        if (EX == 7)  // top byte m, bit j = bit 6 of dim 8j + m
            for (int m = 0; m < 8; ++m) {
                uint8_t b = 0;
                for (int jj = 0; jj < 8; ++jj) b |= (uint8_t)(((v[8 * jj + m] >> 6) & 1) << jj);
                o[48 + m] = b;
            }
    }
    if (g == 0) xipnorm[r] = __fmul_rn(__fmul_rn(ipnorm[r], 2.f), onorm[r]);
}

// FastScan blocks: block b covers rows [vfirst[b], vfirst[b] + vnum[b]) (at
// most 32, zero codes past the end).  Group q (dims 4q..4q+3) is 16 bytes;
// byte j holds vector perm0[j]'s nibble low and vector perm0[j] + 16's high,
// perm0 = {0, 8, 1, 9, ..., 7, 15}, nibble bit 3 = dim 4q.  Then 32 floats of
// ||o - c||.  One thread per output byte of the code part.
__global__ void build_short_kernel(const uint64_t* __restrict__ bits, const float* __restrict__ onorm,
                                   const uint32_t* __restrict__ vfirst, const uint32_t* __restrict__ vnum,
                                   uint64_t nblocks, int D, uint8_t* __restrict__ shrt) {
    const uint64_t code_bytes = 4ull * D, bb = code_bytes + 128;
    const uint64_t total = nblocks * bb;
    const int G = D / 64;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = t / bb;
        const uint32_t rem = (uint32_t)(t - b * bb);
        const uint32_t nv = vnum[b], f = vfirst[b];
        if (rem < code_bytes) {
            const uint32_t q = rem >> 4, jb = rem & 15;
            const uint32_t pv = (jb & 1) ? 8 + (jb >> 1) : (jb >> 1);
            uint8_t byte = 0;
            for (int h = 0; h < 2; ++h) {
                const uint32_t v = pv + 16 * h;
                if (v >= nv) continue;
                const uint64_t w = bits[(size_t)(f + v) * G + (4 * q) / 64];
                const uint32_t s = (4 * q) & 63;
                const uint32_t nib = (uint32_t)(((w >> s) & 1) << 3 | ((w >> (s + 1)) & 1) << 2 |
                                                ((w >> (s + 2)) & 1) << 1 | ((w >> (s + 3)) & 1));
                byte |= (uint8_t)(nib << (4 * h));
            }
            shrt[t] = byte;
        } else {
            const uint32_t v = (rem - (uint32_t)code_bytes) >> 2, by = (rem - (uint32_t)code_bytes) & 3;
            const float fv = v < nv ? onorm[f + v] : 0.f;
            shrt[t] = (uint8_t)(__float_as_uint(fv) >> (8 * by));
        }
    }
}

}  // namespace erq
