/* erq_debug.h - per-stage entry points of liberq.so for parity testing.
 *
 * These run the same kernels as erq_search and copy the intermediate results
 * of one stage back to host memory, so each stage can be compared with the
 * reference on identical inputs.  All buffers are host memory; calls are
 * synchronous on the default stream.
 *
 * Reference stages exposed:
 *   erq_debug_centroid_dists <- L2Sqr16 over all centroids      inc/utils/space.hpp:18-39
 *   erq_debug_probe    <- FlatInitializer::centroids_distances   inc/index/Initializer.hpp:55-68
 *   erq_debug_scan     <- HASearcher::preparing + accumulate_one_block_high_acc's integer
 *                         sums, per probed cluster             inc/index/HASearcher.hpp:121-185,
 *                                                              inc/index/fastscan/FastScan.hpp:214-312
 */
#ifndef ERQ_DEBUG_H
#define ERQ_DEBUG_H

#include "erq.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of int32 entries erq_debug_scan may write for (nq, nprobe). */
ERQ_API uint64_t erq_debug_scan_capacity(const erq_index* index, uint64_t nq, uint64_t nprobe);

/* dist[nq][K]: squared distance of every rotated query to every centroid. */
ERQ_API erq_status erq_debug_centroid_dists(const erq_index* index, const float* rotated_queries,
                                    uint64_t nq, float* dist);

/* cids/sqr_y[nq][nprobe]: probed clusters in ascending distance (ties by id). */
ERQ_API erq_status erq_debug_probe(const erq_index* index, const float* rotated_queries, uint64_t nq,
                           uint64_t nprobe, uint32_t* cids, float* sqr_y);

/* For every (query q, probe rank p): cids, sqr_y, delta (query quantisation
 * step) and sumq (sum of the normalised residual), each [nq][nprobe], and the
 * exact integer sums <x_b, qq> of every vector of the probed cluster, 32 per
 * FastScan block (padding lanes included), starting at S[s_offsets[q][p]].
 * s_capacity must be at least erq_debug_scan_capacity(). */
ERQ_API erq_status erq_debug_scan(const erq_index* index, const float* rotated_queries, uint64_t nq,
                          uint64_t nprobe, uint32_t* cids, float* sqr_y, float* delta,
                          float* sumq, uint64_t* s_offsets, int32_t* S, uint64_t s_capacity);

/* Gradient of the mean cross-entropy of a probe model on host features[n][320]
 * and labels[n], in the parameter order W1[256][320], b1, W2[256][256], b2,
 * W3[8][256], b3 (grads holds ERQ_PROBE_PARAMS floats); loss = mean loss. */
#define ERQ_PROBE_PARAMS 150024
ERQ_API erq_status erq_debug_probe_model_grads(const erq_probe_model* model, const float* features,
                                               const uint8_t* labels, uint64_t n, float* loss,
                                               float* grads);
/* Copies of the FP32 parameters, standardisation and class probe counts
 * (any pointer may be NULL). */
ERQ_API erq_status erq_debug_probe_model_params(const erq_probe_model* model, float* params,
                                                float* mean, float* stdv, uint32_t* bin_nprobe);

/* Polls each pipeline wait of the tcgen05 GEMM makes before it gives up
 * (0 restores the default of 2^26).  A small value makes the waits run out, so
 * a test can check that the GEMM then reports ERQ_ERR_TIMEOUT and leaves the
 * device usable; the GEMM's drain waits (its TMA copies landing, its issued
 * MMAs finishing) always keep the default.  Process-wide. */
ERQ_API erq_status erq_debug_set_gemm_wait_limit(uint32_t polls);

/* C[M][N] = A[M][Kd] * B[N][Kd]^T on the tcgen05 GEMM of the search (BF16
 * operands given as raw 16-bit patterns, FP32 result), host buffers; Kd a
 * multiple of 64.  ERQ_ERR_TIMEOUT if one of its bounded waits ran out. */
ERQ_API erq_status erq_debug_gemm_bf16(const uint16_t* A, const uint16_t* B, uint64_t M, uint64_t N,
                                       uint64_t Kd, float* C, int device);

/* Queries whose coarse probe could not prove its cut from the tensor-core
 * estimates and computed all K exact distances instead, since the last reset
 * (process-wide, per device). */
ERQ_API erq_status erq_debug_probe_fallbacks(int device, uint64_t* count, int reset);

/* Refinement counters since the last call, process-wide per device:
 * stats[0] = exact candidates (vectors whose lower bound was below the top-k
 * threshold at the start of their block: the vectors whose EX-bit distance
 * the reference computes), stats[1] = distances computed (the candidate
 * supersets of the refinement windows), stats[2] = windows, stats[3] =
 * blocks of 32 vectors in those windows.  Waits for the device, returns and
 * resets the counters, and turns counting on or off for refinement launches
 * issued afterwards (a CUDA graph keeps the setting it was captured with). */
ERQ_API erq_status erq_debug_refine_stats(int device, int enable, uint64_t stats[4]);

/* Kernel timing.  While enabled, every kernel launch of the search and
 * rotation entry points is bracketed by CUDA events recorded on the stream
 * the kernel runs on.  erq_profile_read waits for the recorded events and
 * returns, for one kernel ("rotate", "centroid_dist", "select_probe", "scan",
 * "refine", "split", "gemm", "probe", "order", "mlp"), the number of launches and their summed device time since the
 * last reset.  Process-wide; meant for benchmarks. */
ERQ_API void erq_profile_enable(int on);
ERQ_API void erq_profile_reset(void);
ERQ_API erq_status erq_profile_read(const char* kernel, uint64_t* launches, double* total_ms);

#ifdef __cplusplus
}
#endif
#endif /* ERQ_DEBUG_H */
