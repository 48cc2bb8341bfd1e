// Split-BF16 operands for the dense contractions of the path:
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
// The GEMM itself, C[M][N] = A[M][Kd] * B[N][Kd]^T with FP32 accumulation,
// runs on tcgen05 (gemm_tc.cuh); its epilogues are described here.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace erq {

// ----------------------------------------------------------------- split
// out[r][0:Cp] , out[r][Cp:2Cp], out[r][2Cp:3Cp] = (hi, hi, lo) when
// a_side, else (hi, lo, hi); columns >= C of `in` read as 0.  Optionally the
// row's squared norm (float32) into norms[r].  When C and Cp are multiples of
// 8 and both pointers 16-byte aligned, each thread moves 8 columns: two
// float4 loads and three 16-byte stores of 8 bf16; otherwise one column at a
// time.
__device__ __forceinline__ uint32_t pack_bf16x2(__nv_bfloat16 a, __nv_bfloat16 b) {
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

__global__ void split_rows_kernel(const float* __restrict__ in, int R, int C, int Cp,
                                  bool a_side, __nv_bfloat16* __restrict__ out,
                                  float* __restrict__ norms) {
    const int r = blockIdx.x;
    if (r >= R) return;
    const float* src = in + (size_t)r * C;
    __nv_bfloat16* dst = out + (size_t)r * 3 * Cp;
    float nrm = 0.f;
    if (((C | Cp) & 7) == 0 && ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0) {
        for (int c = 8 * threadIdx.x; c < Cp; c += 8 * blockDim.x) {
            float x[8];
            if (c < C) {
                const float4 v0 = reinterpret_cast<const float4*>(src + c)[0];
                const float4 v1 = reinterpret_cast<const float4*>(src + c)[1];
                x[0] = v0.x; x[1] = v0.y; x[2] = v0.z; x[3] = v0.w;
                x[4] = v1.x; x[5] = v1.y; x[6] = v1.z; x[7] = v1.w;
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) x[i] = 0.f;
            }
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const __nv_bfloat16 h0 = __float2bfloat16_rn(x[2 * i]);
                const __nv_bfloat16 h1 = __float2bfloat16_rn(x[2 * i + 1]);
                const __nv_bfloat16 l0 = __float2bfloat16_rn(x[2 * i] - __bfloat162float(h0));
                const __nv_bfloat16 l1 = __float2bfloat16_rn(x[2 * i + 1] - __bfloat162float(h1));
                hi[i] = pack_bf16x2(h0, h1);
                lo[i] = pack_bf16x2(l0, l1);
                nrm = fmaf(x[2 * i], x[2 * i], nrm);
                nrm = fmaf(x[2 * i + 1], x[2 * i + 1], nrm);
            }
            const uint4 H = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            const uint4 L = make_uint4(lo[0], lo[1], lo[2], lo[3]);
            *reinterpret_cast<uint4*>(dst + c) = H;
            *reinterpret_cast<uint4*>(dst + Cp + c) = a_side ? H : L;
            *reinterpret_cast<uint4*>(dst + 2 * Cp + c) = a_side ? L : H;
        }
    } else {
        for (int c = threadIdx.x; c < Cp; c += blockDim.x) {
            const float x = c < C ? src[c] : 0.f;
            const __nv_bfloat16 hi = __float2bfloat16_rn(x);
            const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
            dst[c] = hi;
            dst[Cp + c] = a_side ? hi : lo;
            dst[2 * Cp + c] = a_side ? lo : hi;
            nrm = fmaf(x, x, nrm);
        }
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

// ------------------------------------------------------------- epilogue
// C = acc, or (ranking) C = rn[row] + cn[col] - 2 * acc, or (MLP layers)
// C = acc + bias[col], then max(C, 0) when relu.
struct GemmEpilogue {
    const float* row_norm = nullptr;
    const float* col_norm = nullptr;
    const float* bias = nullptr;
    bool relu = false;
};

}  // namespace erq
