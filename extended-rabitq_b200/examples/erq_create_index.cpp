// erq_create_index - the reference's create_index driver (src/create_index.cpp)
// on liberq.so through the C++ facade include/erq_ivf.hpp: the same input
// files, the same IVF(n, dim, k, b) + construct + save calls, the index built
// on the GPU.
//
//   erq_create_index <data_root> <dataset> <K> <B> [rotation.bin]
//
// Reads <data_root>/<dataset>/<dataset>_base.fvecs, <dataset>_centroid_<K>.fvecs
// and <dataset>_cluster_id_<K>.ivecs (src/create_index.cpp:24-27) and writes
// <data_root>/<dataset>/ivf_exhaf<B>.index.  rotation.bin, when given, holds
// the D x D float32 rotation to use (row-major, as in an index file); without
// it a rotation is drawn from a fixed seed.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "erq_ivf.hpp"

namespace {

template <typename T>
std::vector<T> load_vecs(const std::string& path, size_t& rows, size_t& cols) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    in.seekg(0, std::ios::end);
    const size_t bytes = (size_t)in.tellg();
    in.seekg(0);
    uint32_t c = 0;
    in.read(reinterpret_cast<char*>(&c), 4);
    cols = c;
    rows = bytes / (4 * (cols + 1));
    std::vector<T> out(rows * cols);
    in.seekg(0);
    for (size_t i = 0; i < rows; ++i) {
        in.read(reinterpret_cast<char*>(&c), 4);
        in.read(reinterpret_cast<char*>(&out[i * cols]), 4 * cols);
    }
    return out;
}

}  // namespace

int main(int argc, char* argv[]) {
    if (argc != 5 && argc != 6) {
        std::fprintf(stderr, "usage: %s <data_root> <dataset> <K> <B> [rotation.bin]\n", argv[0]);
        return 2;
    }
    const std::string root = argv[1], ds = argv[2];
    const size_t K = std::strtoull(argv[3], nullptr, 10);
    const int B = std::atoi(argv[4]);
    if (B != 3 && B != 4 && B != 5 && B != 7 && B != 8 && B != 9) {
        std::fprintf(stderr, "B must be 3, 4, 5, 7, 8 or 9\n");
        return 2;
    }
    const std::string dir = root + "/" + ds + "/";
    try {
        size_t N = 0, DIM = 0, kr = 0, kc = 0, nr = 0, nc = 0;
        auto data = load_vecs<float>(dir + ds + "_base.fvecs", N, DIM);
        auto centroids = load_vecs<float>(dir + ds + "_centroid_" + std::to_string(K) + ".fvecs", kr, kc);
        auto cids = load_vecs<uint32_t>(dir + ds + "_cluster_id_" + std::to_string(K) + ".ivecs", nr, nc);
        if (kr != K || kc != DIM || nr != N || nc != 1) {
            std::fprintf(stderr, "input shapes disagree (N=%zu DIM=%zu, centroids %zux%zu, ids %zux%zu)\n",
                         N, DIM, kr, kc, nr, nc);
            return 1;
        }
        std::printf("data loaded\n\tN: %zu\n\tDIM: %zu\n", N, DIM);
        std::vector<float> rot;
        const auto t0 = std::chrono::steady_clock::now();
        erq::IVF ivf(N, DIM, K, (size_t)B);
        ivf.construct(data.data(), centroids.data(), cids.data());
        if (argc == 6) {
            const size_t D = (DIM + 63) / 64 * 64;
            rot.resize(D * D);
            std::ifstream in(argv[5], std::ios::binary);
            if (!in.read(reinterpret_cast<char*>(rot.data()), (std::streamsize)(rot.size() * 4))) {
                std::fprintf(stderr, "%s: expected %zu x %zu float32\n", argv[5], D, D);
                return 1;
            }
            ivf.set_rotation(rot.data());
        }
        ivf.save((dir + "ivf_exhaf" + std::to_string(B) + ".index").c_str());
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("ivf constructed and saved\nIndexing time: %.3f s\n", s);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
