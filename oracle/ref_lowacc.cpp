// Oracle harness over the reference's non-HIGH_ACC path (test
// infrastructure): the same unmodified headers as ref_harness.cpp compiled
// WITHOUT HIGH_ACC_FAST_SCAN, so that IVF builds and reads the 4-factor
// block format (inc/index/Quantizer.hpp:33-37, 290-300) and searches with
// Searcher (inc/index/Searcher.hpp).  The reference's drivers always define
// HIGH_ACC_FAST_SCAN; this harness is how that second format is produced and
// searched here.  Exposes a C ABI for the Python tests.
#include <bits/stdc++.h>
#include <immintrin.h>
#include <omp.h>

#define EIGEN_DONT_PARALLELIZE
#define private public
#include "index/IVF.hpp"
#undef private

namespace {
struct CoutSilencer {
    std::streambuf* old;
    std::ofstream null;
    CoutSilencer() : old(std::cout.rdbuf()), null("/dev/null") { std::cout.rdbuf(null.rdbuf()); }
    ~CoutSilencer() { std::cout.rdbuf(old); }
};
struct LowAccIndex {
    IVF ivf;
};
}  // namespace

extern "C" {

// IVF(n, dim, K, bits) + construct + save, as src/create_index.cpp:45-49 does.
int lref_build(const float* data, uint64_t n, uint64_t dim, const float* centroids, uint64_t K,
               const uint32_t* cluster_ids, uint64_t bits, const char* path) {
    CoutSilencer quiet;
    IVF ivf(n, dim, K, bits);
    ivf.construct(data, centroids, cluster_ids);
    ivf.save(path);
    return 0;
}

void* lref_load(const char* path) {
    std::ifstream probe(path, std::ios::binary);
    if (!probe.is_open()) return nullptr;
    probe.close();
    auto* r = new LowAccIndex();
    CoutSilencer quiet;
    r->ivf.load(path);
    return r;
}

void lref_free(void* h) { delete static_cast<LowAccIndex*>(h); }

void lref_info(void* h, uint64_t* out) {
    const IVF& ivf = static_cast<LowAccIndex*>(h)->ivf;
    out[0] = ivf.N;
    out[1] = ivf.DIM;
    out[2] = ivf.D;
    out[3] = ivf.K;
    out[4] = ivf.EX_BITS;
}

void lref_rotate(void* h, const float* q, uint64_t nq, float* qrot) {
    const IVF& ivf = static_cast<LowAccIndex*>(h)->ivf;
    FloatRowMat in(nq, ivf.D), out(nq, ivf.D);
    in.setZero();
    for (uint64_t i = 0; i < nq; ++i) std::memcpy(&in(i, 0), q + i * ivf.DIM, sizeof(float) * ivf.DIM);
    ivf.Rota.rotate(in, out);
    std::memcpy(qrot, out.data(), sizeof(float) * nq * ivf.D);
}

// IVF::search (inc/index/IVF.hpp:295-324 with Searcher) for each query,
// returning the pool's ids and distances (unfilled: id 0, +inf).
void lref_search_dists(void* h, const float* qrot, uint64_t nq, uint64_t k, uint64_t nprobe,
                       uint32_t* ids, float* dists) {
    const IVF& ivf = static_cast<LowAccIndex*>(h)->ivf;
    for (uint64_t q = 0; q < nq; ++q) {
        const float* query = qrot + q * ivf.D;
        std::vector<Candidate> centroid_dist(nprobe);
        ivf.initer->centroids_distances(query, nprobe, centroid_dist);
        ResultPool KNNs(k);
        Searcher searcher(query, ivf.D, ivf.EX_BITS, ivf.DQ);
        for (size_t i = 0; i < nprobe; ++i) {
            PID cid = centroid_dist[i].id;
            searcher.search_cluster(ivf.ClusterLst[cid], ivf.initer->centroid(cid),
                                    centroid_dist[i].distance, KNNs);
        }
        KNNs.copy_results(ids + q * k);
        for (size_t i = 0; i < k; ++i)
            dists[q * k + i] = i < KNNs.size_ ? KNNs.distances_[i] : std::numeric_limits<float>::infinity();
    }
}

}  // extern "C"
