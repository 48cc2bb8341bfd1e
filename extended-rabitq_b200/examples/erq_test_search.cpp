// erq_test_search - the reference's test_search driver (src/test_search.cpp)
// on liberq.so through the C++ facade include/erq_ivf.hpp.
//
//   erq_test_search <data_root> <dataset> <B> [results.csv]
//
// Reads <data_root>/<dataset>/<dataset>_{base,query}.fvecs,
// <dataset>_groundtruth.ivecs and ivf_exhaf<B>.index (the file names of
// src/test_search.cpp:35-39), rotates the queries, chooses the nprobe list the
// way get_nprobes does (src/test_search.cpp:155-199), and writes
// nprobe,QPS,recall,ratio averaged over 3 rounds (src/test_search.cpp:101-150).
// Unlike the reference, each nprobe's queries go to the GPU in one batch; QPS
// is NQ / (rotation + search wall time).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <queue>
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

double l2(const float* a, const float* b, size_t n) {
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += (double(a[i]) - b[i]) * (double(a[i]) - b[i]);
    return s;
}

// get_ratio (inc/utils/tools.hpp:16-51)
double get_ratio(const float* q, const float* base, size_t dim, const uint32_t* gt,
                 const uint32_t* res, size_t k) {
    std::priority_queue<double> g, a;
    for (size_t i = 0; i < k; ++i) {
        g.emplace(l2(q, base + (size_t)gt[i] * dim, dim));
        a.emplace(l2(q, base + (size_t)res[i] * dim, dim));
    }
    double ret = 0;
    size_t valid = 0;
    while (!g.empty()) {
        if (g.top() > 1e-5) {
            ret += std::sqrt(a.top() / g.top());
            ++valid;
        }
        g.pop();
        a.pop();
    }
    return valid == 0 ? 1.0 * k : ret / valid * k;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <data_root> <dataset> <B> [results.csv]\n", argv[0]);
        return 2;
    }
    const std::string root = argv[1], ds = argv[2];
    const int B = std::atoi(argv[3]);
    const std::string dir = root + "/" + ds + "/";
    const std::string csv = argc > 4 ? argv[4] : ds + "_exhaf" + std::to_string(B) + ".csv";
    const size_t TOPK = 100, ROUND = 3;
    try {
        size_t nb, dim, nq, qdim, ng, gcols;
        auto base = load_vecs<float>(dir + ds + "_base.fvecs", nb, dim);
        auto query = load_vecs<float>(dir + ds + "_query.fvecs", nq, qdim);
        auto gt = load_vecs<uint32_t>(dir + ds + "_groundtruth.ivecs", ng, gcols);
        if (qdim != dim || ng < nq || gcols < TOPK) throw std::runtime_error("inconsistent inputs");

        erq::IVF ivf;
        ivf.load((dir + "ivf_exhaf" + std::to_string(B) + ".index").c_str());
        const size_t D = ivf.padded_dim();
        std::vector<float> rotated(nq * D);
        auto t0 = std::chrono::steady_clock::now();
        ivf.rotator().rotate(query.data(), nq, rotated.data());
        const double rotate_s =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

        std::vector<size_t> all = {5};
        for (size_t i = 10; i < 200; i += 10) all.push_back(i);
        for (size_t i = 200; i < 400; i += 40) all.push_back(i);
        for (size_t i = 400; i <= 1500; i += 100) all.push_back(i);
        for (size_t i = 2000; i <= 4000; i += 500) all.push_back(i);
        all.push_back(6000);
        all.push_back(10000);
        all.push_back(15000);

        std::vector<uint32_t> res(nq * TOPK);
        auto recall_of = [&]() {
            size_t correct = 0;
            for (size_t i = 0; i < nq; ++i)
                for (size_t j = 0; j < TOPK; ++j)
                    for (size_t k = 0; k < TOPK; ++k)
                        if (gt[i * gcols + k] == res[i * TOPK + j]) {
                            ++correct;
                            break;
                        }
            return double(correct) / double(nq * TOPK);
        };
        // get_nprobes: stop past recall 0.997 or when recall stops improving
        std::vector<size_t> nprobes;
        double old_recall = 0;
        for (size_t np : all) {
            if (np > ivf.k()) break;
            nprobes.push_back(np);
            ivf.search_batch(rotated.data(), nq, TOPK, np, res.data());
            const double r = recall_of();
            if (r > 0.997 || r - old_recall < 1e-5) break;
            std::printf("%g\t%zu\n", r, np);
            old_recall = r;
        }
        std::ofstream out(csv);
        out << "nprobe,QPS,recall,ratio\n";
        for (size_t np : nprobes) {
            double qps = 0, recall = 0, ratio = 0;
            for (size_t r = 0; r < ROUND; ++r) {
                auto s0 = std::chrono::steady_clock::now();
                ivf.search_batch(rotated.data(), nq, TOPK, np, res.data());
                const double sec =
                    std::chrono::duration<double>(std::chrono::steady_clock::now() - s0).count();
                qps += nq / (sec + rotate_s);
                recall += recall_of();
                double tr = 0;
                for (size_t i = 0; i < nq; ++i)
                    tr += get_ratio(&query[i * dim], base.data(), dim, &gt[i * gcols],
                                    &res[i * TOPK], TOPK);
                ratio += tr / double(nq * TOPK);
            }
            out << np << ',' << qps / ROUND << ',' << recall / ROUND << ',' << ratio / ROUND << '\n';
        }
        std::printf("wrote %s\n", csv.c_str());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
