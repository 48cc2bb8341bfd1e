// Stand-in for the HNSW graph library header that the Extended-RaBitQ reference
// includes (inc/index/Initializer.hpp:11).  Test infrastructure only.
//
// The reference uses HNSW only for the coarse quantiser when K >= 20000
// (inc/index/IVF.hpp:157-161); every workload here has K <= 16384, so the
// flat initializer is always selected.  These types exist so the reference
// headers compile; any attempt to use them aborts.
#pragma once

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <queue>
#include <string>
#include <utility>

namespace hnswlib {

using labeltype = size_t;

[[noreturn]] inline void hnsw_unavailable() {
    std::fprintf(stderr, "HNSW coarse quantiser (K >= 20000) is not available in this build\n");
    std::abort();
}

class L2Space {
   public:
    explicit L2Space(size_t dim) : dim_(dim) {}

   private:
    size_t dim_;
};

template <typename dist_t>
class HierarchicalNSW {
   public:
    HierarchicalNSW(L2Space*, size_t, size_t = 16, size_t = 200) { hnsw_unavailable(); }
    void addPoint(const void*, labeltype) { hnsw_unavailable(); }
    char* getDataByInternalId(size_t) const { hnsw_unavailable(); }
    void setEf(size_t) { hnsw_unavailable(); }
    std::priority_queue<std::pair<dist_t, labeltype>> searchKnn(const void*, size_t) const {
        hnsw_unavailable();
    }
    void saveIndex(const std::string&) { hnsw_unavailable(); }
    void loadIndex(const std::string&, L2Space*, size_t) { hnsw_unavailable(); }
};

}  // namespace hnswlib
