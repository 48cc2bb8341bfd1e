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
