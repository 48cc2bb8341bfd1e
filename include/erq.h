/* erq.h - C ABI of the B200 IVF search for Extended-RaBitQ indexes.
 *
 * The library (extended-rabitq_b200/lib/liberq.so) loads an index file written
 * by the reference's IVF::save and answers IVF::search queries on one GPU.
 * Every entry point takes plain pointers and sizes; pointers may be host or
 * device memory (detected per pointer).  No entry point aborts: errors come
 * back as erq_status codes with a message from erq_last_error().
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   erq_index_load   <- IVF::load            inc/index/IVF.hpp:254-293
 *   erq_index_get_info <- IVF::padded_dim / IVF::k and the header fields
 *                                            inc/index/IVF.hpp:86-90,261-265
 *   erq_rotate       <- Rotator::rotate       inc/index/Rotator.hpp:60-63, with the
 *                       query padding of src/test_search.cpp:83-92
 *   erq_search       <- IVF::search           inc/index/IVF.hpp:295-324
 *   erq_search_raw   <- the rotate-then-search sequence of src/test_search.cpp:83-110
 *   erq_index_free   <- IVF::~IVF             inc/index/IVF.hpp:106
 */
#ifndef ERQ_H
#define ERQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ERQ_API_VERSION 1

#if defined(__GNUC__)
#define ERQ_API __attribute__((visibility("default")))
#else
#define ERQ_API
#endif

typedef enum erq_status {
    ERQ_OK = 0,
    ERQ_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, k, nprobe, ... */
    ERQ_ERR_IO = 2,               /* index file cannot be opened or read */
    ERQ_ERR_FORMAT = 3,           /* header or sizes inconsistent, file truncated */
    ERQ_ERR_UNSUPPORTED = 4,      /* e.g. K >= 20000 (HNSW side file), D > 2048 */
    ERQ_ERR_CUDA = 5,             /* a CUDA runtime call failed */
    ERQ_ERR_OUT_OF_MEMORY = 6,    /* device or host allocation failed */
    ERQ_ERR_TIMEOUT = 7           /* a bounded device-side wait gave up */
} erq_status;

typedef struct erq_index erq_index;

typedef struct erq_index_info {
    uint64_t n;            /* number of data vectors (N) */
    uint64_t dim;          /* raw dimension (DIM) */
    uint64_t padded_dim;   /* D = DIM rounded up to a multiple of 64 */
    uint64_t num_clusters; /* K */
    uint64_t ex_bits;      /* EX_BITS = total bits - 1, one of 2,3,4,6,7,8 */
    uint64_t device_bytes; /* device memory held by the index */
    int device;            /* CUDA device ordinal */
    int block_factors;     /* factors per vector in a FastScan block: 1 (the reference
                              drivers' HIGH_ACC_FAST_SCAN format) or 4 (its format
                              without that define, searched as inc/index/Searcher.hpp) */
} erq_index_info;

/* Library version (ERQ_API_VERSION) and status text. */
ERQ_API int erq_version(void);
ERQ_API const char* erq_status_string(erq_status s);
/* Message of the last failing call on this thread ("" if none). */
ERQ_API const char* erq_last_error(void);

/* Load an index file (the reference's IVF::save format) onto CUDA device
 * `device`.  Reads both block formats the reference
 * writes (one factor per vector with HIGH_ACC_FAST_SCAN, four without; told
 * apart by the file size).  Any K: for K >= 20000 the reference probes with an
 * HNSW graph from a side file, which is not read here - the probe stays exact
 * (the Flat semantics, inc/index/Initializer.hpp:55-68).  Rejects D > 2048. */
ERQ_API erq_status erq_index_load(const char* path, int device, erq_index** out);
ERQ_API erq_status erq_index_get_info(const erq_index* index, erq_index_info* info);
ERQ_API void erq_index_free(erq_index* index);

/* rotated[nq][D] = pad(queries[nq][DIM]) * P, as test_search does before
 * calling IVF::search.  `stream` is a cudaStream_t (NULL: default stream). */
ERQ_API erq_status erq_rotate(const erq_index* index, const float* queries, uint64_t nq,
                      float* rotated, void* stream);

/* IVF::search for nq rotated queries (each D floats, row-major).
 * ids[nq][k]: result ids in ascending estimated distance, exactly as the
 *   reference's ResultPool::copy_results (unfilled slots are 0).
 * dists[nq][k] (may be NULL): the pool's distance estimates; unfilled slots
 *   are +inf.
 * Requires 1 <= nprobe <= K and 1 <= k <= 1024.  The result equals the
 * reference's on the same index and query bytes.  When any pointer is host
 * memory the call returns after the results are in host memory; with device
 * pointers only it is asynchronous on `stream`. */
ERQ_API erq_status erq_search(const erq_index* index, const float* rotated_queries, uint64_t nq,
                      uint64_t k, uint64_t nprobe, uint32_t* ids, float* dists, void* stream);

/* Rotate then search: queries are raw DIM-float vectors. */
ERQ_API erq_status erq_search_raw(const erq_index* index, const float* queries, uint64_t nq,
                          uint64_t k, uint64_t nprobe, uint32_t* ids, float* dists,
                          void* stream);

/* ---------------------------------------------------------------------------
 * Learned probing.  Has no counterpart in the reference (IVF::search probes a
 * fixed nprobe, inc/index/IVF.hpp:295-324).  A small MLP predicts, per query,
 * after how many clusters of its probe list the plain search's top-k stops
 * changing; the search then scans only those clusters, with the reference's
 * arithmetic unchanged.  Training uses labels produced by the plain search. */
typedef struct erq_probe_model erq_probe_model;
#define ERQ_PROBE_FEATURES 320 /* 256 sketch dims + 64 nearest-centroid terms */
#define ERQ_PROBE_BINS 8

/* features[nq][320] of rotated queries: the first 256 rotated coordinates
 * scaled by 16/||q||, log(e_0/||q||^2) and e_j/e_0 - 1 (j = 1..63) of the 64
 * nearest exact centroid distances e_0 <= e_1 <= ... */
ERQ_API erq_status erq_probe_features(const erq_index* index, const float* rotated_queries,
                                      uint64_t nq, float* features, void* stream);

/* Train on host features[n][320] and labels[n] in [0, 8); bin_nprobe[8]
 * (increasing) is the probe count of each class.  Adam, cross-entropy,
 * mini-batches of `batch`, on CUDA device `device`. */
ERQ_API erq_status erq_probe_model_train(const float* features, const uint8_t* labels, uint64_t n,
                                         const uint32_t* bin_nprobe, int epochs, int batch,
                                         float lr, uint64_t seed, int device,
                                         erq_probe_model** out, float* final_loss);
ERQ_API erq_status erq_probe_model_save(const erq_probe_model* model, const char* path);
ERQ_API erq_status erq_probe_model_load(const char* path, int device, erq_probe_model** out);
ERQ_API void erq_probe_model_free(erq_probe_model* model);
/* probs[n][8] = softmax of the model on raw features[n][320]. */
ERQ_API erq_status erq_probe_model_predict(const erq_probe_model* model, const float* features,
                                           uint64_t n, float* probs, void* stream);

/* IVF::search where each query scans the first c clusters of its probe list:
 * c = bin_nprobe of the smallest class whose cumulative probability reaches
 * `confidence`, or nprobe_fallback when the most likely class has probability
 * below `min_prob`.  nprobe_used[nq] (may be NULL) receives c per query.  The
 * results equal erq_search's with nprobe = c for each query. */
ERQ_API erq_status erq_search_learned(const erq_index* index, const erq_probe_model* model,
                                      const float* rotated_queries, uint64_t nq, uint64_t k,
                                      uint64_t nprobe_fallback, float confidence, float min_prob,
                                      uint32_t* ids, float* dists, uint32_t* nprobe_used,
                                      void* stream);

/* The same with raw DIM-float queries, rotated inside (test_search's sequence). */
ERQ_API erq_status erq_search_learned_raw(const erq_index* index, const erq_probe_model* model,
                                          const float* queries, uint64_t nq, uint64_t k,
                                          uint64_t nprobe_fallback, float confidence,
                                          float min_prob, uint32_t* ids, float* dists,
                                          uint32_t* nprobe_used, void* stream);

/* ---------------------------------------------------------------------------
 * Batched search plans.  No counterpart in the reference, which searches one
 * query at a time (IVF::search, inc/index/IVF.hpp:295-324); a plan returns the
 * same ids and distances as erq_search (plain) or erq_search_learned (with a
 * model) for every query of a batch.
 *
 * A plan owns every device buffer a batch of up to max_batch queries needs, so
 * erq_plan_search allocates nothing.  The first search of each batch size
 * captures the pipeline (rotation when raw_queries, coarse probe, learned
 * cut-off when a model is given, work list, scan, refinement) into a CUDA
 * graph that later searches of that size replay.  The scan runs over a work
 * list of (cluster, up to Q queries probing it, chunk of up to C 32-vector
 * blocks) items in one persistent kernel; erq_plan_autotune times the tile
 * choices on a sample batch and keeps the fastest for that batch size.
 * Calls on one plan are serialised by the plan; use one plan per stream for
 * concurrent batches. */
typedef struct erq_plan erq_plan;

typedef struct {
    uint32_t queries_per_item;  /* Q: 1, 2 or 4 queries sharing one cluster chunk */
    uint32_t blocks_per_item;   /* C: cluster chunk, in 32-vector blocks */
    uint32_t warps;             /* warps per scan block: 4 or 8 */
    uint32_t refine_warps;      /* refinement form: 4 (a block of 4 warps per query, windows
                                   of 16 blocks), 32 (the wide form, windows of 128 blocks),
                                   or 0 = 32 when the batch has no more queries than SMs,
                                   else 4 */
} erq_plan_tuning;

/* model may be NULL (plain fixed-nprobe search); with a model, nprobe is the
 * fallback probe count.  raw_queries: queries are DIM floats and are rotated
 * inside, else they are rotated D floats. */
ERQ_API erq_status erq_plan_create(const erq_index* index, const erq_probe_model* model,
                                   uint64_t max_batch, uint64_t k, uint64_t nprobe,
                                   int raw_queries, erq_plan** out);
ERQ_API void erq_plan_free(erq_plan* plan);
/* Confidence and minimum probability of the learned cut-off (defaults 0.9, 0). */
ERQ_API erq_status erq_plan_set_learned(erq_plan* plan, float confidence, float min_prob);
/* Times every tile choice on queries[n] (host or device; best of `reps` runs
 * each), then both refinement forms with the fastest tile, and keeps the
 * fastest for batches of about n queries. */
ERQ_API erq_status erq_plan_autotune(erq_plan* plan, const float* queries, uint64_t n, int reps,
                                     erq_plan_tuning* chosen, float* best_ms);
ERQ_API erq_status erq_plan_set_tuning(erq_plan* plan, uint64_t batch, const erq_plan_tuning* tuning);
/* The tuning a batch of `batch` queries uses (the nearest tuned size, else a default). */
ERQ_API erq_status erq_plan_get_tuning(const erq_plan* plan, uint64_t batch, erq_plan_tuning* tuning);
/* Searches queries[nq] (nq <= max_batch).  Buffers may be host or device
 * memory; with any host buffer the call returns when the results are in,
 * otherwise it is asynchronous on `stream`.  dists and nprobe_used may be NULL. */
ERQ_API erq_status erq_plan_search(erq_plan* plan, const float* queries, uint64_t nq, uint32_t* ids,
                                   float* dists, uint32_t* nprobe_used, void* stream);
/* Device bytes the plan holds. */
ERQ_API uint64_t erq_plan_device_bytes(const erq_plan* plan);
/* on = 0 launches the kernels one by one instead of replaying a graph (same
 * results; lets the kernel profiler of erq_debug.h time each launch). */
ERQ_API erq_status erq_plan_set_graphs(erq_plan* plan, int on);
/* How erq_plan_search runs a batch with host buffers: as `chunks` pieces
 * whose host-to-device copies, searches and device-to-host copies overlap
 * (two buffer slots, two copy streams); 1 (the default) for one piece, 0 for
 * 4 pieces from 8192 queries and 2 from 4096.  Results are the same in every
 * case. */
ERQ_API erq_status erq_plan_set_pipeline(erq_plan* plan, int chunks);
/* erq_plan_search that returns without waiting, also with host buffers: the
 * queries are copied in on the plan's copy stream into one of two buffer
 * slots (alternating between calls), the search and the copy of the results
 * out run on `stream`.  So the copy-in of a call overlaps the search of the
 * one before.  Host buffers must be pinned for the copies to overlap; the
 * queries must stay unchanged and the results must not be read until
 * `stream` has been synchronised.  Results equal erq_plan_search's. */
ERQ_API erq_status erq_plan_search_async(erq_plan* plan, const float* queries, uint64_t nq,
                                         uint32_t* ids, float* dists, uint32_t* nprobe_used,
                                         void* stream);

/* ---------------------------------------------------------------------------
 * IVF clustering.  Replaces the reference's offline clustering step
 * (python/ivf.py:5-34, faiss IVF{K},Flat training = Lloyd's k-means with
 * random initial centroids drawn from the data and empty clusters re-seeded
 * by splitting a populated one), whose centroid and cluster-id files feed
 * create_index.  Distances on the tensor cores (split-BF16, about FP32
 * accuracy), centroid sums in 64-bit fixed point (deterministic: the same
 * seed gives the same clusters), splitmix64 as the random stream.  Buffers
 * may be host or device memory; the calls are synchronous. */

/* k-means of data[n][dim] into k clusters: `iters` Lloyd iterations from k
 * distinct random points, then a last assignment.  centroids: [k][dim];
 * assign (optional): [n], the nearest final centroid of each point. */
ERQ_API erq_status erq_kmeans(const float* data, uint64_t n, uint64_t dim, uint64_t k, int iters,
                              uint64_t seed, float* centroids, uint32_t* assign, int device);
/* One Lloyd iteration from centroids_in: assign[n] (nearest centroid, ties to
 * the smaller index), counts[k] (cluster sizes of that assignment),
 * centroids_out = the means, then the empty clusters split with the random
 * stream started at `seed`. */
ERQ_API erq_status erq_kmeans_step(const float* data, uint64_t n, uint64_t dim, uint64_t k,
                                   const float* centroids_in, uint64_t seed,
                                   float* centroids_out, uint32_t* assign, uint32_t* counts,
                                   int device);

/* ---------------------------------------------------------------------------
 * Index construction on the GPU: IVF(n, dim, k, total_bits) + construct +
 * save (inc/index/IVF.hpp:116-153, 219-252; src/create_index.cpp:45-49),
 * HIGH_ACC_FAST_SCAN format.  data[n][dim], centroids[k][dim] (raw, as
 * create_index reads them), cluster_ids[n] < k; buffers host or device.
 * `rotation` (D x D row-major, D = dim rounded up to 64; queries are rotated
 * as q * rotation) may be NULL, in which case a random orthogonal matrix is
 * drawn from `seed`.  Given the same rotation, the file equals the
 * reference's byte for byte, except the block factors of the lanes past a
 * cluster's end, which the reference leaves unset and this writes as 0.
 * Every step follows the reference's arithmetic (see build.cuh).  Synchronous. */
ERQ_API erq_status erq_build_index(const float* data, uint64_t n, uint64_t dim,
                                   const float* centroids, uint64_t k, const uint32_t* cluster_ids,
                                   uint64_t total_bits, const float* rotation, uint64_t seed,
                                   const char* path, int device);

/* erq_search without any memory allocation.  Has no counterpart in the
 * reference: it is for callers that cannot allocate device memory while a
 * query runs - engines that hand all GPU memory to their own allocator up
 * front, or serving loops that forbid allocation on the request path - and
 * so cannot let erq_search take its scratch from a memory pool.
 *
 * All pointers must be device memory (queries 16-byte aligned, ids/dists
 * 4-byte aligned); the call is asynchronous on `stream`.  The pipeline's
 * scratch is a fixed 64 MiB array in the library's device memory, held on
 * every GPU that loads the library until the process exits.  A request that
 * does not fit (about nq * (4K + 128 * blocks of the nprobe largest clusters)
 * bytes) fails with ERQ_ERR_INVALID_ARGUMENT and a message giving the largest
 * batch that fits.  The first call on a device looks up the array's device
 * address and keeps it for the life of the process, so the library must not
 * be used across a cudaDeviceReset of that device; make that first call
 * before any stream capture.  Every call uses
 * the same array: calls that overlap on the GPU (different streams, or
 * different threads without ordering) race and must be serialised by the
 * caller.  Results equal erq_search's. */
ERQ_API erq_status erq_search_noalloc(const erq_index* index, const float* rotated_queries,
                                      uint64_t nq, uint64_t k, uint64_t nprobe, uint32_t* ids,
                                      float* dists, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ERQ_H */
