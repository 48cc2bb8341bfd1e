// Shared device helpers for the Extended-RaBitQ IVF search kernels (sm_100a).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace erq {

constexpr int kFastSize = 32;     // vectors per FastScan block (inc/defines.hpp:13)
constexpr int kMaxD = 2048;       // u16 lane sums of the reference are exact up to here
constexpr int kMaxTopK = 1024;    // largest k the refine kernel's pool supports
constexpr float kNormEps = 1e-5f; // normalize_query16's eps (inc/utils/space.hpp:756)
constexpr float kConstBound = 0.58f;  // inc/index/fastscan/FastScan.hpp:295

// Sum of 16 lane partials held by lanes 0..15 of a half-warp, combined in the
// order GCC 13 expands _mm512_reduce_add_ps: (l, l+8), (l, l+4), (0,2)/(1,3),
// then the last pair.  shfl_down by 8,4,2,1 inside a 16-lane segment performs
// exactly those pairings (float addition is commutative, so a+b == b+a
// bitwise).  The result is valid in lane 0 of the segment.
__device__ __forceinline__ float tree16_sum(float v) {
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 8, 16));
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 4, 16));
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 2, 16));
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 1, 16));
    return v;
}

// Packed FP32 pairs (sm_100a f32x2): two independent IEEE round-to-nearest
// operations per instruction, each equal to its scalar counterpart.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;"
        : "=l"(d)
        : "l"(*reinterpret_cast<const uint64_t*>(&a)), "l"(*reinterpret_cast<const uint64_t*>(&b)),
          "l"(*reinterpret_cast<const uint64_t*>(&c)));
    return *reinterpret_cast<float2*>(&d);
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(d)
        : "l"(*reinterpret_cast<const uint64_t*>(&a)), "l"(*reinterpret_cast<const uint64_t*>(&b)));
    return *reinterpret_cast<float2*>(&d);
}

// (float)(1.0 / (double)x): the reference computes these reciprocals in
// double and rounds once to float (inc/utils/space.hpp:760,774;
// inc/index/HASearcher.hpp:56).
__device__ __forceinline__ float recip_via_double(float x) {
    return __double2float_rn(__ddiv_rn(1.0, (double)x));
}

// (int16_t)(t + 0.5 - (t < 0)) evaluated in double (high_acc_quantize16,
// inc/utils/space.hpp:708-709).  For |t| <= 8191 the double sum is exact, so
// this is round-half-away-from-zero of t.
__device__ __forceinline__ int quantize_round(float t) {
    return (int)__double2int_rz(__dadd_rn(__dadd_rn((double)t, 0.5), t < 0.f ? -1.0 : 0.0));
}

// Orderable 64-bit key of (non-negative float distance, id): ascending keys
// are ascending distance, ties by ascending id.
__device__ __forceinline__ uint64_t dist_key(float d, uint32_t id) {
    return ((uint64_t)__float_as_uint(d) << 32) | id;
}

__host__ __device__ __forceinline__ uint64_t div_up(uint64_t a, uint64_t b) {
    return (a + b - 1) / b;
}

// Lower bound of one vector's distance (accumulate_one_block_high_acc,
// inc/index/fastscan/FastScan.hpp:295-323): constants of the (query, cluster)
// pair, then lb = ((ipq - c1) * c2 * onorm + c3) + onorm^2 in that order.
struct LbConsts {
    float c1, c2, c3;
};
__device__ __forceinline__ LbConsts lb_consts(float sumq, float y, float one_over_sqrtD) {
    LbConsts k;
    k.c1 = __double2float_rn(__dsub_rn(__dmul_rn(0.5, (double)sumq), (double)kConstBound));
    k.c2 = __fmul_rn(__fmul_rn(-5.f, y), one_over_sqrtD);
    k.c3 = __fmul_rn(y, y);
    return k;
}
__device__ __forceinline__ float lower_bound(float ipq, float on, const LbConsts& k) {
    float t = __fsub_rn(ipq, k.c1);
    t = __fmul_rn(t, k.c2);
    t = __fmul_rn(t, on);
    t = __fadd_rn(t, k.c3);
    return __fadd_rn(t, __fmul_rn(on, on));
}
// Smallest lower bound of a 32-vector block over a warp (lane = vector;
// invalid lanes pass +inf); valid in every lane.
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

}  // namespace erq
