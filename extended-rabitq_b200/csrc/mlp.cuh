// Learned probing: a small MLP that predicts, per query, how many clusters the
// plain search must probe before its top-k stops changing.
//
//   features (320) -> 256 -> ReLU -> 256 -> ReLU -> 8 logits -> softmax
//
// Weights are kept as FP32 master copies for training and as BF16 copies for
// the forward pass; every product accumulates in FP32.  The forward, backward
// and Adam kernels are written here (no library).  The model only chooses how
// many of the probe list's clusters each query scans; the distance arithmetic
// of the search is unchanged.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace erq {

constexpr int kMlpIn = 320;      // 256 sketch dims + 64 centroid distances
constexpr int kMlpHidden = 256;
constexpr int kMlpBins = 8;
constexpr int kSketchDims = 256;
constexpr int kFeatDists = 64;

// Parameter layout (one flat FP32 array; the BF16 copy mirrors W1, W2, W3).
constexpr int kW1 = 0;                                  // [256][320]
constexpr int kB1 = kW1 + kMlpHidden * kMlpIn;          // [256]
constexpr int kW2 = kB1 + kMlpHidden;                   // [256][256]
constexpr int kB2 = kW2 + kMlpHidden * kMlpHidden;      // [256]
constexpr int kW3 = kB2 + kMlpHidden;                   // [8][256]
constexpr int kB3 = kW3 + kMlpBins * kMlpHidden;        // [8]
constexpr int kMlpParams = kB3 + kMlpBins;

// C[m][n] (+)= sum_k A(m,k) * B(k,n) with A(m,k) = A[m*sam + k*sak] and
// B(k,n) = B[k*sbk + n*sbn]; 16x16 tiles through shared memory.  TB is float
// or __nv_bfloat16.  Optional bias[n] and ReLU on the result.
template <typename TB>
__global__ void mlp_matmul_kernel(const float* __restrict__ A, long sam, long sak,
                                  const TB* __restrict__ B, long sbk, long sbn,
                                  float* __restrict__ C, int M, int N, int K,
                                  const float* __restrict__ bias, bool relu, bool accumulate) {
    __shared__ float As[16][17];
    __shared__ float Bs[16][17];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m = blockIdx.y * 16 + ty, n = blockIdx.x * 16 + tx;
    float acc = 0.f;
    for (int k0 = 0; k0 < K; k0 += 16) {
        const int ka = k0 + tx, kb = k0 + ty;
        const int am = blockIdx.y * 16 + ty, bn = blockIdx.x * 16 + tx;
        As[ty][tx] = (am < M && ka < K) ? A[am * sam + (long)ka * sak] : 0.f;
        float bv = 0.f;
        if (kb < K && bn < N) {
            if constexpr (sizeof(TB) == 2)
                bv = __bfloat162float(B[(long)kb * sbk + (long)bn * sbn]);
            else
                bv = (float)B[(long)kb * sbk + (long)bn * sbn];
        }
        Bs[ty][tx] = bv;
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) acc = fmaf(As[ty][kk], Bs[kk][tx], acc);
        __syncthreads();
    }
    if (m < M && n < N) {
        float v = acc + (bias ? bias[n] : 0.f);
        if (relu) v = fmaxf(v, 0.f);
        C[(size_t)m * N + n] = accumulate ? C[(size_t)m * N + n] + v : v;
    }
}

// Softmax cross-entropy on logits [B][8]: dlogits = (softmax - onehot) / B,
// probabilities out, per-row loss into loss_rows.
__global__ void mlp_softmax_xent_kernel(const float* __restrict__ logits,
                                        const uint8_t* __restrict__ labels, int B,
                                        float* __restrict__ probs, float* __restrict__ dlogits,
                                        float* __restrict__ loss_rows) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B) return;
    const float* z = logits + (size_t)r * kMlpBins;
    float mx = z[0];
    for (int j = 1; j < kMlpBins; ++j) mx = fmaxf(mx, z[j]);
    float e[kMlpBins], s = 0.f;
    for (int j = 0; j < kMlpBins; ++j) {
        e[j] = expf(z[j] - mx);
        s += e[j];
    }
    const float inv = 1.f / s;
    for (int j = 0; j < kMlpBins; ++j) {
        const float p = e[j] * inv;
        if (probs) probs[(size_t)r * kMlpBins + j] = p;
        if (dlogits) dlogits[(size_t)r * kMlpBins + j] = (p - (labels && labels[r] == j ? 1.f : 0.f)) / B;
    }
    if (loss_rows && labels) loss_rows[r] = -(z[labels[r]] - mx - logf(s));
}

// Output layer and softmax of inference in one pass: z = h2 . W3^T + b3 and
// probs = softmax(z).  Eight threads per row (one per bin), 32 rows per block
// of 256; each dot product runs k = 0..255 in order and the softmax sums the
// bins in order, so the results equal mlp_matmul_kernel followed by
// mlp_softmax_xent_kernel.  W3 (BF16 [8][256]) is staged in shared memory as
// floats, bin-minor, so the 8 threads of a row read consecutive banks.
__global__ void __launch_bounds__(256) mlp_head_kernel(const float* __restrict__ h2,
                                                       const __nv_bfloat16* __restrict__ w3,
                                                       const float* __restrict__ b3, int B,
                                                       float* __restrict__ probs) {
    __shared__ float ws[kMlpHidden * kMlpBins];
    for (int i = threadIdx.x; i < kMlpHidden * kMlpBins; i += blockDim.x) {
        const int j = i / kMlpHidden, k = i - j * kMlpHidden;
        ws[k * kMlpBins + j] = __bfloat162float(w3[i]);
    }
    __syncthreads();
    const int r = blockIdx.x * (blockDim.x / kMlpBins) + threadIdx.x / kMlpBins;
    const int j = threadIdx.x % kMlpBins;
    float acc = 0.f;
    if (r < B) {
        const float4* h = reinterpret_cast<const float4*>(h2 + (size_t)r * kMlpHidden);
#pragma unroll 4
        for (int k4 = 0; k4 < kMlpHidden / 4; ++k4) {
            const float4 v = h[k4];
            acc = fmaf(v.x, ws[(4 * k4 + 0) * kMlpBins + j], acc);
            acc = fmaf(v.y, ws[(4 * k4 + 1) * kMlpBins + j], acc);
            acc = fmaf(v.z, ws[(4 * k4 + 2) * kMlpBins + j], acc);
            acc = fmaf(v.w, ws[(4 * k4 + 3) * kMlpBins + j], acc);
        }
    }
    const float zj = acc + b3[j];
    float z[kMlpBins];
#pragma unroll
    for (int t = 0; t < kMlpBins; ++t) z[t] = __shfl_sync(0xffffffffu, zj, t, kMlpBins);
    float mx = z[0];
    for (int t = 1; t < kMlpBins; ++t) mx = fmaxf(mx, z[t]);
    float s = 0.f, ej = 0.f;
    for (int t = 0; t < kMlpBins; ++t) {
        const float e = expf(z[t] - mx);
        s += e;
        if (t == j) ej = e;
    }
    if (r < B) probs[(size_t)r * kMlpBins + j] = ej * (1.f / s);
}

// dH *= (H > 0), elementwise.
__global__ void mlp_relu_grad_kernel(float* __restrict__ dH, const float* __restrict__ H, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && H[i] <= 0.f) dH[i] = 0.f;
}

// db[n] = sum_r dY[r][n]
__global__ void mlp_bias_grad_kernel(const float* __restrict__ dY, int B, int N,
                                     float* __restrict__ db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int r = 0; r < B; ++r) s += dY[(size_t)r * N + n];
    db[n] = s;
}

// Adam on the FP32 master weights, refreshing the BF16 copies of W1..W3.
__global__ void mlp_adam_kernel(float* __restrict__ w, const float* __restrict__ g,
                                float* __restrict__ m1, float* __restrict__ m2,
                                __nv_bfloat16* __restrict__ wb, int n, float lr, float beta1,
                                float beta2, float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = beta1 * m1[i] + (1.f - beta1) * gi;
    const float b = beta2 * m2[i] + (1.f - beta2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float v = w[i] - lr * (a / bc1) / (sqrtf(b / bc2) + eps);
    w[i] = v;
    wb[i] = __float2bfloat16_rn(v);
}

__global__ void mlp_to_bf16_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb,
                                   int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// Standardise raw features: x = (f - mean) / std.
__global__ void mlp_standardise_kernel(const float* __restrict__ f, const float* __restrict__ mean,
                                       const float* __restrict__ stdv, float* __restrict__ x,
                                       int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int c = i % kMlpIn;
        x[i] = (f[i] - mean[c]) / stdv[c];
    }
}

// Tensor-core inference.  Activations x (FP32) are split as x = hi + lo with
// hi = bf16(x), lo = bf16(x - hi), written [hi | lo] per row; the weights are
// duplicated as [W | W], so one BF16 GEMM with FP32 accumulation gives
// hi.W + lo.W, x.W to within 2^-16 relative (the BF16 weights are exact).
__device__ __forceinline__ void split2(float x, __nv_bfloat16* hi, __nv_bfloat16* lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    *hi = h;
    *lo = __float2bfloat16_rn(x - __bfloat162float(h));
}

// xs[r] = [hi | lo] of (f[r] - mean) / std, 2 * kMlpIn columns.
__global__ void mlp_standardise_split_kernel(const float* __restrict__ f, const float* __restrict__ mean,
                                             const float* __restrict__ stdv,
                                             __nv_bfloat16* __restrict__ xs, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = i / kMlpIn, c = i - r * kMlpIn;
    const float x = (f[i] - mean[c]) / stdv[c];
    split2(x, xs + (size_t)r * 2 * kMlpIn + c, xs + (size_t)r * 2 * kMlpIn + kMlpIn + c);
}

// hs[r] = [hi | lo] of h[r], 2 * kMlpHidden columns.
__global__ void mlp_split_hidden_kernel(const float* __restrict__ h, __nv_bfloat16* __restrict__ hs,
                                        int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = i / kMlpHidden, c = i - r * kMlpHidden;
    split2(h[i], hs + (size_t)r * 2 * kMlpHidden + c, hs + (size_t)r * 2 * kMlpHidden + kMlpHidden + c);
}

// w1d = [W1 | W1] ([256][640]), w2d = [W2 | W2] ([256][512]) from the BF16 copy.
__global__ void mlp_dup_weights_kernel(const __nv_bfloat16* __restrict__ wb,
                                       __nv_bfloat16* __restrict__ w1d,
                                       __nv_bfloat16* __restrict__ w2d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kMlpHidden * 2 * kMlpIn) {
        const int r = i / (2 * kMlpIn), c = (i - r * 2 * kMlpIn) % kMlpIn;
        w1d[i] = wb[kW1 + r * kMlpIn + c];
    }
    if (i < kMlpHidden * 2 * kMlpHidden) {
        const int r = i / (2 * kMlpHidden), c = (i - r * 2 * kMlpHidden) % kMlpHidden;
        w2d[i] = wb[kW2 + r * kMlpHidden + c];
    }
}

// Raw features of one query: 256 sketch dims (the first rotated coordinates,
// a random projection, scaled by 16/||q_r||) and 64 values of its nearest
// centroid distances e_0 <= e_1 <= ... (the tensor-core estimates, FP32
// accurate): log(e_0 / ||q_r||^2 + 1e-12) and e_j / e_0 - 1 for j >= 1.
// With xs, the standardised features (f - mean) / std are also written as
// [hi | lo] BF16, the input of the first layer (mlp_standardise_split_kernel's
// arithmetic).
// qnorm: the squared norms of the rotated queries when already computed
// (the split kernel's), else each block sums its row.
__global__ void probe_features_kernel(const float* __restrict__ qrot, int D,
                                      const float* __restrict__ qnorm,
                                      const float* __restrict__ near_d, int nq,
                                      float* __restrict__ feats, const float* __restrict__ mean,
                                      const float* __restrict__ stdv,
                                      __nv_bfloat16* __restrict__ xs) {
    const int q = blockIdx.x;
    if (q >= nq) return;
    const float* v = qrot + (size_t)q * D;
    float qn;
    if (qnorm) {
        qn = qnorm[q];
    } else {
        __shared__ float red[8];
        float s = 0.f;
        for (int i = threadIdx.x; i < D; i += blockDim.x) s = fmaf(v[i], v[i], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        qn = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) qn += red[w];
    }
    const float inv = qn > 0.f ? 16.f / sqrtf(qn) : 0.f;
    float* f = feats + (size_t)q * kMlpIn;
    __nv_bfloat16* xr = xs ? xs + (size_t)q * 2 * kMlpIn : nullptr;
    auto put = [&](int c, float x) {
        f[c] = x;
        if (xr) split2((x - mean[c]) / stdv[c], xr + c, xr + kMlpIn + c);
    };
    for (int i = threadIdx.x; i < kSketchDims; i += blockDim.x) put(i, i < D ? v[i] * inv : 0.f);
    const float* d = near_d + (size_t)q * kFeatDists;
    const float d0 = d[0];
    for (int j = threadIdx.x; j < kFeatDists; j += blockDim.x) {
        float x;
        if (j == 0)
            x = logf(d0 / fmaxf(qn, 1e-30f) + 1e-12f);
        else
            x = d0 > 0.f ? d[j] / d0 - 1.f : 0.f;
        put(kSketchDims + j, x);
    }
}

// Per-query probe count from the class probabilities: the smallest bin whose
// cumulative probability reaches `confidence`; queries whose most likely bin
// has probability below `min_prob` fall back to `fallback`.
__global__ void mlp_choose_nprobe_kernel(const float* __restrict__ probs, int nq,
                                         const int* __restrict__ bin_nprobe, float confidence,
                                         float min_prob, int fallback, int nprobe_cap,
                                         int* __restrict__ q_nprobe) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const float* p = probs + (size_t)q * kMlpBins;
    float mx = 0.f, cum = 0.f;
    int chosen = -1;
    for (int j = 0; j < kMlpBins; ++j) {
        mx = fmaxf(mx, p[j]);
        cum += p[j];
        if (chosen < 0 && cum >= confidence) chosen = j;
    }
    int np = (chosen < 0 || mx < min_prob) ? fallback : bin_nprobe[chosen];
    q_nprobe[q] = min(max(np, 1), nprobe_cap);
}

}  // namespace erq
