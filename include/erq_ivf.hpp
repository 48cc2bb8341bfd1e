// erq_ivf.hpp - C++ facade of liberq.so with the reference's IVF interface.
//
// Header-only; link with -lerq (extended-rabitq_b200/lib/liberq.so).  The class
// keeps the names, argument meaning and call pattern of the reference's IVF
// (inc/index/IVF.hpp:62-127) and Rotator (inc/index/Rotator.hpp:9-63) so host
// code written against them (src/test_search.cpp) keeps its structure:
//
//   IVF ivf;  ivf.load(path);                      // IVF::load
//   ivf.rotator().rotate(queries, nq, rotated);     // Rotator::rotate
//   ivf.search(&rotated[i * D], nullptr, k, nprobe, results);   // IVF::search
//
// Differences a caller sees:
//   * rotate also takes raw row-major buffers (the matrix form accepts any
//     row-major matrix type with rows()/cols()/data(), Eigen's FloatRowMat
//     included, with the output already sized rows x D);
//   * errors throw erq::Error (the reference asserts or aborts);
//   * search_batch answers many queries in one call (the GPU's fast path);
//   * building keeps the reference's calls (IVF(n, dim, k, b), construct,
//     save; src/create_index.cpp:45-49) but runs at save(): construct only
//     records its three pointers, which must stay valid until then, and
//     set_rotation may fix the rotation (else one is drawn from a seed).
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "erq.h"

namespace erq {

class Error : public std::runtime_error {
   public:
    Error(erq_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    erq_status status;
};

inline void check(erq_status s) {
    if (s != ERQ_OK) throw Error(s, std::string(erq_status_string(s)) + ": " + erq_last_error());
}

class IVF;

// Rotator::rotate over raw buffers: rotated[nq][D] = pad(queries[nq][DIM]) * P.
class Rotator {
   public:
    void rotate(const float* queries, size_t nq, float* rotated, void* stream = nullptr) const {
        check(erq_rotate(index_, queries, nq, rotated, stream));
    }

    // Rotator::rotate(const FloatRowMat& A, FloatRowMat& RAND_A)
    // (inc/index/Rotator.hpp:60-63): RAND_A = A * P for row-major matrices.
    // A holds one query per row, DIM columns or already zero-padded to D
    // (src/test_search.cpp:83-90 passes the padded form); RAND_A must be
    // rows x D, as test_search allocates it.
    template <class Mat>
    void rotate(const Mat& A, Mat& RAND_A) const {
        const size_t nq = static_cast<size_t>(A.rows());
        const size_t cols = static_cast<size_t>(A.cols());
        if (cols != DIM_ && cols != D_)
            throw Error(ERQ_ERR_INVALID_ARGUMENT, "rotate: matrix has " + std::to_string(cols) +
                                                      " columns; expected DIM or padded D");
        if (static_cast<size_t>(RAND_A.rows()) != nq || static_cast<size_t>(RAND_A.cols()) != D_)
            throw Error(ERQ_ERR_INVALID_ARGUMENT, "rotate: output must be rows x padded D");
        if (cols == DIM_) {
            rotate(A.data(), nq, RAND_A.data());
            return;
        }
        // padded input: the columns past DIM are zero, so rotate the first DIM
        std::vector<float> q(nq * DIM_);
        for (size_t i = 0; i < nq; ++i)
            std::memcpy(&q[i * DIM_], A.data() + i * cols, DIM_ * sizeof(float));
        rotate(q.data(), nq, RAND_A.data());
    }
    size_t size() const;

   private:
    friend class IVF;
    const erq_index* index_ = nullptr;
    size_t D_ = 0;
    size_t DIM_ = 0;
};

inline size_t Rotator::size() const { return D_; }

class IVF {
   public:
    IVF() = default;
    explicit IVF(int device) : device_(device) {}
    // IVF(n, dim, k, b) (inc/index/IVF.hpp:116-153): an index to be built.
    IVF(size_t n, size_t dim, size_t k, size_t total_bits, int device = 0)
        : device_(device), build_n_(n), build_dim_(dim), build_k_(k), build_bits_(total_bits) {}
    IVF(const IVF&) = delete;
    IVF& operator=(const IVF&) = delete;
    ~IVF() { erq_index_free(index_); }

    // IVF::load (inc/index/IVF.hpp:254-293)
    void load(const char* filename) {
        erq_index* idx = nullptr;
        check(erq_index_load(filename, device_, &idx));
        erq_index_free(index_);
        index_ = idx;
        check(erq_index_get_info(index_, &info_));
        rot_.index_ = index_;
        rot_.D_ = info_.padded_dim;
        rot_.DIM_ = info_.dim;
    }

    // IVF::search (inc/index/IVF.hpp:295-324): one rotated query (D floats);
    // `data` is unused, as in the reference; results gets k ids.
    void search(const float* query, const float* data, size_t k, size_t nprobe,
                uint32_t* results) const {
        (void)data;
        check(erq_search(index_, query, 1, k, nprobe, results, nullptr, nullptr));
    }

    // Many rotated queries at once (host or device buffers); dists may be null.
    void search_batch(const float* queries, size_t nq, size_t k, size_t nprobe, uint32_t* ids,
                      float* dists = nullptr, void* stream = nullptr) const {
        check(erq_search(index_, queries, nq, k, nprobe, ids, dists, stream));
    }

    // IVF::construct (inc/index/IVF.hpp:155-217): data[n][dim], centroids[k][dim]
    // (raw), cluster_ids[n]; host or device pointers, kept until save().
    void construct(const float* data, const float* centroids, const uint32_t* cluster_ids) {
        if (!build_n_) throw Error(ERQ_ERR_INVALID_ARGUMENT, "construct: use IVF(n, dim, k, b)");
        data_ = data;
        centroids_ = centroids;
        cluster_ids_ = cluster_ids;
    }
    // The rotation to use (D x D row-major, D = dim rounded up to 64), in
    // place of one drawn from `seed`; the file then equals the reference's
    // for the same rotation.  Kept by pointer until save().
    void set_rotation(const float* rotation, uint64_t seed = 0) {
        rotation_ = rotation;
        seed_ = seed;
    }
    // IVF::save (inc/index/IVF.hpp:219-252): quantises on the GPU
    // (erq_build_index) and writes the index file.
    void save(const char* filename) const {
        if (!data_) throw Error(ERQ_ERR_INVALID_ARGUMENT, "save: nothing constructed");
        check(erq_build_index(data_, build_n_, build_dim_, centroids_, build_k_, cluster_ids_,
                              build_bits_, rotation_, seed_, filename, device_));
    }

    size_t padded_dim() const { return info_.padded_dim; }  // IVF::padded_dim
    size_t k() const { return info_.num_clusters; }         // IVF::k
    size_t size() const { return info_.n; }
    size_t dim() const { return info_.dim; }
    Rotator& rotator() { return rot_; }                      // IVF::rotator

   private:
    int device_ = 0;
    erq_index* index_ = nullptr;
    erq_index_info info_{};
    Rotator rot_;
    // build side
    size_t build_n_ = 0, build_dim_ = 0, build_k_ = 0, build_bits_ = 0;
    const float* data_ = nullptr;
    const float* centroids_ = nullptr;
    const uint32_t* cluster_ids_ = nullptr;
    const float* rotation_ = nullptr;
    uint64_t seed_ = 0;
};

}  // namespace erq
