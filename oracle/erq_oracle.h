/* CPU oracle for the Extended-RaBitQ IVF search path (test infrastructure).
 *
 * A plain-C restatement of the reference's query path, used only by the tests,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker.
 * It is never linked into, or called by, the product library.
 *
 * Every function cites the reference code it restates (paths relative to the
 * reference project root).  Floating-point steps follow the reference's
 * evaluation order exactly: 16-lane accumulations in dimension order reduced by
 * the same pairwise tree GCC uses for _mm512_reduce_add_ps, explicit fused
 * multiply-adds where the reference uses _mm512_fmadd_ps, and double precision
 * where the reference's expressions promote to double.  This file must be
 * compiled with -ffp-contract=off and without -ffast-math.
 */
#ifndef ERQ_ORACLE_H
#define ERQ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_index orc_index;

/* Parse an index file written by the reference's IVF::save
 * (inc/index/IVF.hpp:219-252).  Returns 0 on success, a negative code on
 * error: -1 open/read, -2 bad header, -3 cluster sizes do not sum to N,
 * -4 unsupported (K >= 20000 needs the HNSW side file), -5 truncated, -6 OOM. */
int orc_index_load(const char* path, orc_index** out);
void orc_index_free(orc_index* idx);
/* out[0..4] = N, DIM, D, K, EX_BITS */
void orc_index_info(const orc_index* idx, uint64_t* out);
/* raw views (owned by the index) */
const float* orc_centroids(const orc_index* idx);
const float* orc_rotation(const orc_index* idx);
const uint64_t* orc_cluster_sizes(const orc_index* idx);

/* L2Sqr16 (inc/utils/space.hpp:18-39) */
float orc_l2sqr16(const float* x, const float* y, uint64_t L);

/* FlatInitializer::centroids_distances (inc/index/Initializer.hpp:55-68);
 * ties in distance are ordered by ascending cluster id. */
void orc_probe(const orc_index* idx, const float* q, uint64_t nprobe, uint32_t* cids,
               float* sqr_y);

/* HASearcher::preparing (inc/index/HASearcher.hpp:121-185): unit_q[D], qq[D],
 * delta, sumq and the un-shifted 16-entry group tables lut[D/4*16]. */
void orc_prepare(uint64_t D, const float* q, const float* c, float sqr_y, float* unit_q,
                 int16_t* qq, float* delta, float* sumq, int32_t* lut);

/* Exact <x_b, qq> for the 32 vectors of one FastScan block
 * (inc/index/fastscan/FastScan.hpp:214-308). */
void orc_block_sums(uint64_t D, const uint8_t* block_codes, const int32_t* lut, int32_t* S);

/* Scan every block of cluster `cid` for query q at a fixed distk:
 * S, ipq (=float(S)*delta) per lane and the raw lower-bound mask per block
 * (inc/index/fastscan/FastScan.hpp:295-323).  Returns the block count. */
uint64_t orc_scan_cluster(const orc_index* idx, const float* q, uint32_t cid, float sqr_y,
                          float distk, int32_t* S, float* ipq, uint32_t* masks);

/* Decode one vector's EX-bit code (layouts of store_compacted_code,
 * inc/index/Quantizer.hpp:491-631) into D byte values. */
void orc_ex_decode(uint64_t D, uint64_t EX, const uint8_t* code, uint8_t* out);
/* IP_FUNC(unit_q, code) (inc/utils/space.hpp IP*_fxu*) */
float orc_ex_ip(uint64_t D, uint64_t EX, const float* unit_q, const uint8_t* code);
/* the EX code of the vector at position pos (cluster order) */
const uint8_t* orc_long_code(const orc_index* idx, uint64_t pos);

/* IVF::search (inc/index/IVF.hpp:295-324) for one rotated query.  ids as
 * ResultPool::copy_results (unfilled slots 0); dists may be NULL (unfilled
 * slots +inf). */
void orc_search(const orc_index* idx, const float* q, uint64_t k, uint64_t nprobe,
                uint32_t* ids, float* dists);
/* Many queries; nthreads > 1 spreads them over OpenMP threads. */
void orc_search_batch(const orc_index* idx, const float* q, uint64_t nq, uint64_t k,
                      uint64_t nprobe, uint32_t* ids, float* dists, int nthreads);
/* Every refined candidate (id, ex_dist) in the order it is offered to the
 * top-k pool; returns the total count (entries past cap are dropped). */
uint64_t orc_trace(const orc_index* idx, const float* q, uint64_t k, uint64_t nprobe,
                   uint64_t cap, uint32_t* cand_ids, float* cand_dist);

#ifdef __cplusplus
}
#endif
#endif
