// C ABI of the B200 IVF search (include/erq.h, include/erq_debug.h).
//
// Host side: parse the reference's index file (IVF::load,
// inc/index/IVF.hpp:254-293), place it in device memory in the layout of
// layout.cuh, and drive the search pipeline of IVF::search
// (inc/index/IVF.hpp:295-324) over batches of queries:
//
//   centroid_dist_kernel -> probe_exact_kernel -> scan_kernel -> refine_kernel
//
// Per-call scratch comes from the stream-ordered allocator on the caller's
// stream, so concurrent calls on different streams never share workspace.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cmath>
#include <numeric>
#include <random>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/erq.h"
#include "../../include/erq_debug.h"
#include "coarse.cuh"
#include "gemm.cuh"
#include "build.cuh"
#include "gemm_tc.cuh"
#include "kmeans.cuh"
#include "mlp.cuh"
#include "probe.cuh"
#include "layout.cuh"
#include "lowacc.cuh"
#include "refine.cuh"
#include "order.cuh"
#include "scan.cuh"
#include "scan_batch.cuh"

using namespace erq;

// probe selection sorts all K centroid keys in shared memory (8 bytes each)
constexpr uint64_t kMaxClusters = 1ull << 24;

// ------------------------------------------------------------------ errors
namespace {
thread_local std::string g_last_error;

erq_status fail(erq_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

#define ERQ_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            return fail(e_ == cudaErrorMemoryAllocation ? ERQ_ERR_OUT_OF_MEMORY : ERQ_ERR_CUDA, \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                        __LINE__);                                                        \
        }                                                                                 \
    } while (0)

#define ERQ_TRY(expr)                  \
    do {                               \
        erq_status s_ = (expr);        \
        if (s_ != ERQ_OK) return s_;   \
    } while (0)

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    erq_status set(int dev) {
        ERQ_CUDA(cudaGetDevice(&prev));
        if (prev != dev) ERQ_CUDA(cudaSetDevice(dev));
        return ERQ_OK;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

bool is_device_ptr(const void* p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();  // clear
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// Stream-ordered scratch allocations (from the index's memory pool) released
// on scope exit.
struct Scratch {
    cudaStream_t stream;
    cudaMemPool_t pool;
    std::vector<void*> ptrs;
    Scratch(cudaStream_t s, cudaMemPool_t p) : stream(s), pool(p) {}
    template <typename T>
    erq_status alloc(T** out, size_t count) {
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
        cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, stream);
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? ERQ_ERR_OUT_OF_MEMORY : ERQ_ERR_CUDA,
                        "cudaMallocAsync(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return ERQ_OK;
    }
    ~Scratch() {
        for (void* p : ptrs) cudaFreeAsync(p, stream);
    }
};

// ----------------------------------------------------------------- profiler
// Event pairs around kernel launches, resolved lazily by erq_profile_read.
enum KernelId {
    kRotate = 0,
    kCentroidDist,
    kSelectProbe,
    kScan,
    kRefine,
    kSplit,
    kGemm,
    kProbe,
    kOrder,
    kMlp,
    kNumKernels
};
const char* const kKernelNames[kNumKernels] = {"rotate", "centroid_dist", "select_probe", "scan",
                                               "refine", "split",  "gemm",          "probe",
                                               "order", "mlp"};

struct Profiler {
    std::mutex mu;
    bool on = false;
    struct Rec {
        int kernel;
        int device;
        cudaEvent_t start, stop;
    };
    std::vector<Rec> pending;
    uint64_t launches[kNumKernels] = {};
    double ms[kNumKernels] = {};
};
Profiler& profiler() {
    static Profiler p;
    return p;
}

// Records the start event on construction and the stop event on finish().
struct LaunchTimer {
    int kernel;
    cudaStream_t stream;
    cudaEvent_t start = nullptr, stop = nullptr;
    bool active = false;
    LaunchTimer(int k, cudaStream_t s) : kernel(k), stream(s) {
        Profiler& p = profiler();
        {
            std::lock_guard<std::mutex> g(p.mu);
            active = p.on;
        }
        if (!active) return;
        // launches recorded into a CUDA graph are not timed one by one
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            active = false;
            return;
        }
        if (cudaEventCreate(&start) != cudaSuccess || cudaEventCreate(&stop) != cudaSuccess) {
            active = false;
            return;
        }
        cudaEventRecord(start, stream);
    }
    void finish() {
        if (!active) return;
        cudaEventRecord(stop, stream);
        int dev = 0;
        cudaGetDevice(&dev);
        Profiler& p = profiler();
        std::lock_guard<std::mutex> g(p.mu);
        p.pending.push_back({kernel, dev, start, stop});
        active = false;
    }
};

}  // namespace

// ------------------------------------------------------------------- index
struct erq_index {
    int device = 0;
    uint64_t N = 0, DIM = 0, D = 0, K = 0, EX = 0;
    uint64_t total_blocks = 0;
    uint64_t device_bytes = 0;
    std::vector<uint32_t> h_nblocks;     // per cluster
    std::vector<uint64_t> top_blocks;    // top_blocks[p] = blocks of the p largest clusters
    // device arrays
    float* P = nullptr;
    float* centroids = nullptr;
    uint8_t* codes = nullptr;
    float* onorm = nullptr;
    uint8_t* excode = nullptr;      // device layout, ex_row bytes per vector
    uint64_t ex_row = 0;
    float* xipnorm = nullptr;
    uint32_t* ids = nullptr;
    // 4 factors per vector: the reference's format without HIGH_ACC_FAST_SCAN
    // (onorm then holds ||o - c||^2; lowacc.cuh)
    int factors = 1;
    float* fac_ip = nullptr;
    float* fac_sumxb = nullptr;
    float* fac_err = nullptr;
    uint32_t* c_first_block = nullptr;
    uint32_t* c_first_vec = nullptr;
    uint32_t* c_size = nullptr;
    uint32_t* c_nblocks = nullptr;
    uint32_t* c_size_rank = nullptr;  // [K] rank of each cluster by decreasing size (ties by id)
    uint32_t* c_by_size = nullptr;    // [K] the clusters by decreasing size (ties by id)
    // split-BF16 operands of the tensor-core GEMMs (gemm.cuh)
    __nv_bfloat16* c_split = nullptr;   // [K][3D] centroids (hi | lo | hi)
    __nv_bfloat16* pt_split = nullptr;  // [D][3D] rows of P^T (hi | lo | hi)
    float* cn = nullptr;                // [K] squared centroid norms
    float* c_chain = nullptr;           // [K][D] centroids in chain order (probe.cuh)
    float cn_max = 0.f;
    float eps_rel = 0.f;                // distance-estimate bound (probe.cuh)
    // per-call scratch pool; keeps freed blocks for reuse by later calls
    cudaMemPool_t pool = nullptr;

    ~erq_index() {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (pool) {
            cudaDeviceSynchronize();
            cudaMemPoolDestroy(pool);
        }
        for (void* p : {(void*)P, (void*)centroids, (void*)codes, (void*)onorm, (void*)excode,
                        (void*)xipnorm, (void*)ids, (void*)c_first_block, (void*)c_first_vec,
                        (void*)c_size, (void*)c_nblocks, (void*)c_size_rank, (void*)c_by_size, (void*)c_split,
                        (void*)pt_split,
                        (void*)cn, (void*)c_chain, (void*)fac_ip, (void*)fac_sumxb, (void*)fac_err})
            if (p) cudaFree(p);
        if (prev >= 0) cudaSetDevice(prev);
    }
};

namespace {

struct FileCloser {
    void operator()(FILE* f) const {
        if (f) fclose(f);
    }
};

erq_status read_to_device(FILE* f, void* dst, size_t bytes, std::vector<uint8_t>& staging,
                          const char* what) {
    const size_t chunk = staging.size();
    uint8_t* d = static_cast<uint8_t*>(dst);
    for (size_t off = 0; off < bytes; off += chunk) {
        const size_t n = std::min(chunk, bytes - off);
        if (fread(staging.data(), 1, n, f) != n)
            return fail(ERQ_ERR_FORMAT, "index file truncated while reading %s", what);
        ERQ_CUDA(cudaMemcpy(d + off, staging.data(), n, cudaMemcpyHostToDevice));
    }
    return ERQ_OK;
}

template <typename T>
erq_status dev_alloc(erq_index* idx, T** p, size_t count) {
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? ERQ_ERR_OUT_OF_MEMORY : ERQ_ERR_CUDA,
                    "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    idx->device_bytes += bytes;
    return ERQ_OK;
}

erq_status load_impl(const char* path, erq_index* idx) {
    std::unique_ptr<FILE, FileCloser> f(fopen(path, "rb"));
    if (!f) return fail(ERQ_ERR_IO, "cannot open index file '%s'", path);
    uint64_t hdr[4];
    if (fread(hdr, sizeof(uint64_t), 4, f.get()) != 4)
        return fail(ERQ_ERR_FORMAT, "index file '%s' too short for its header", path);
    idx->N = hdr[0];
    idx->DIM = hdr[1];
    idx->K = hdr[2];
    idx->EX = hdr[3];
    const uint64_t EX = idx->EX;
    if (!(EX == 2 || EX == 3 || EX == 4 || EX == 6 || EX == 7 || EX == 8))
        return fail(ERQ_ERR_FORMAT, "unsupported EX_BITS %llu (expected 2,3,4,6,7,8)",
                    (unsigned long long)EX);
    if (idx->DIM == 0 || idx->K == 0)
        return fail(ERQ_ERR_FORMAT, "bad header: DIM=%llu K=%llu", (unsigned long long)idx->DIM,
                    (unsigned long long)idx->K);
    // K >= 20000: the reference loads an HNSW graph over the centroids from a
    // side file (inc/index/IVF.hpp:157-161, 274-291) and probes approximately;
    // this library ignores the side file and probes every K exactly (the
    // Flat path's semantics, inc/index/Initializer.hpp:55-68).
    if (idx->K > kMaxClusters)
        return fail(ERQ_ERR_UNSUPPORTED, "K=%llu exceeds the %llu clusters the probe selection supports",
                    (unsigned long long)idx->K, (unsigned long long)kMaxClusters);
    idx->D = (idx->DIM + 63) / 64 * 64;
    if (idx->D > (uint64_t)kMaxD)
        return fail(ERQ_ERR_UNSUPPORTED, "padded dimension %llu exceeds %d",
                    (unsigned long long)idx->D, kMaxD);
    if (idx->N >= (1ull << 32))
        return fail(ERQ_ERR_UNSUPPORTED, "N=%llu exceeds 2^32-1", (unsigned long long)idx->N);
    const uint64_t D = idx->D, K = idx->K, N = idx->N;

    std::vector<uint64_t> sizes(K);
    if (fread(sizes.data(), sizeof(uint64_t), K, f.get()) != K)
        return fail(ERQ_ERR_FORMAT, "index file truncated in the cluster sizes");
    std::vector<uint32_t> first_block(K), first_vec(K), csize(K);
    idx->h_nblocks.resize(K);
    uint64_t tot = 0, blocks = 0;
    for (uint64_t c = 0; c < K; ++c) {
        if (sizes[c] > N) return fail(ERQ_ERR_FORMAT, "cluster %llu larger than N", (unsigned long long)c);
        first_block[c] = (uint32_t)blocks;
        first_vec[c] = (uint32_t)tot;
        csize[c] = (uint32_t)sizes[c];
        idx->h_nblocks[c] = (uint32_t)div_up(sizes[c], kFastSize);
        tot += sizes[c];
        blocks += idx->h_nblocks[c];
    }
    if (tot != N)
        return fail(ERQ_ERR_FORMAT, "cluster sizes sum to %llu, header says N=%llu",
                    (unsigned long long)tot, (unsigned long long)N);
    idx->total_blocks = blocks;
    {
        std::vector<uint64_t> nbs(idx->h_nblocks.begin(), idx->h_nblocks.end());
        std::sort(nbs.begin(), nbs.end(), std::greater<uint64_t>());
        idx->top_blocks.assign(K + 1, 0);
        for (uint64_t i = 0; i < K; ++i) idx->top_blocks[i + 1] = idx->top_blocks[i] + nbs[i];
    }
    // The remaining bytes - P, centroids, short data, long codes, factors,
    // ids - tell the two block formats apart: 1 factor per vector
    // (HIGH_ACC_FAST_SCAN, the reference drivers' format) or 4.
    const uint64_t code_len = D * EX / 8;
    {
        const long here = ftell(f.get());
        if (here < 0 || fseek(f.get(), 0, SEEK_END) != 0)
            return fail(ERQ_ERR_IO, "cannot size index file '%s'", path);
        const uint64_t rest = (uint64_t)ftell(f.get()) - (uint64_t)here;
        if (fseek(f.get(), here, SEEK_SET) != 0) return fail(ERQ_ERR_IO, "seek failed in '%s'", path);
        auto need = [&](uint64_t F) {
            return (D * D + K * D) * 4 + blocks * (4 * D + kFastSize * 4 * F) + N * (code_len + 8);
        };
        if (rest == need(1)) idx->factors = 1;
        else if (rest == need(4)) idx->factors = 4;
        else if (K >= 20000 && (rest == need(1) - K * D * 4 || rest == need(4) - K * D * 4))
            return fail(ERQ_ERR_UNSUPPORTED,
                        "index file '%s' (K=%llu) keeps its centroids only in the reference's "
                        "hnswlib side file, which this library does not read; indexes written by "
                        "erq_build_index carry them in the main file", path, (unsigned long long)K);
        else
            return fail(ERQ_ERR_FORMAT, "index file '%s' holds %llu bytes after its cluster table; "
                        "%llu (one block factor) or %llu (four) expected", path,
                        (unsigned long long)rest, (unsigned long long)need(1),
                        (unsigned long long)need(4));
    }
    const uint64_t raw_block = 4 * D + kFastSize * sizeof(float) * idx->factors;

    std::vector<uint8_t> staging(64ull << 20);
    ERQ_TRY(dev_alloc(idx, &idx->P, D * D));
    ERQ_TRY(read_to_device(f.get(), idx->P, D * D * sizeof(float), staging, "the rotation matrix"));
    ERQ_TRY(dev_alloc(idx, &idx->centroids, K * D));
    ERQ_TRY(read_to_device(f.get(), idx->centroids, K * D * sizeof(float), staging, "the centroids"));
    {
        uint8_t* raw = nullptr;
        cudaError_t e = cudaMalloc(&raw, std::max<uint64_t>(blocks * raw_block, 16));
        if (e != cudaSuccess) return fail(ERQ_ERR_OUT_OF_MEMORY, "cudaMalloc for short codes failed");
        erq_status s = read_to_device(f.get(), raw, blocks * raw_block, staging, "the short codes");
        if (s == ERQ_OK) s = dev_alloc(idx, &idx->codes, blocks * code_block_bytes((int)D));
        if (s == ERQ_OK) s = dev_alloc(idx, &idx->onorm, blocks * kFastSize);
        if (s == ERQ_OK && idx->factors == 4) s = dev_alloc(idx, &idx->fac_ip, blocks * kFastSize);
        if (s == ERQ_OK && idx->factors == 4) s = dev_alloc(idx, &idx->fac_sumxb, blocks * kFastSize);
        if (s == ERQ_OK && idx->factors == 4) s = dev_alloc(idx, &idx->fac_err, blocks * kFastSize);
        if (s == ERQ_OK && blocks > 0) {
            float* extra[3] = {idx->fac_ip, idx->fac_sumxb, idx->fac_err};
            transform_blocks_kernel<<<1184, 256>>>(raw, idx->codes, idx->onorm, blocks, (int)D,
                                                   idx->factors, idx->factors == 4 ? 4 : 2,
                                                   extra[0], extra[1], extra[2]);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
            if (e != cudaSuccess)
                s = fail(ERQ_ERR_CUDA, "block layout kernel failed: %s", cudaGetErrorString(e));
        }
        cudaFree(raw);
        if (s != ERQ_OK) return s;
    }
    idx->ex_row = ex_row_bytes((int)D, (int)EX);
    ERQ_TRY(dev_alloc(idx, &idx->excode, std::max<uint64_t>(N * idx->ex_row, 64)));
    {
        uint8_t* raw = nullptr;
        cudaError_t e = cudaMalloc(&raw, std::max<uint64_t>(N * code_len, 16));
        if (e != cudaSuccess) return fail(ERQ_ERR_OUT_OF_MEMORY, "cudaMalloc for EX-bit codes failed");
        erq_status s = read_to_device(f.get(), raw, N * code_len, staging, "the EX-bit codes");
        if (s == ERQ_OK && N > 0) {
            uint32_t* dst = reinterpret_cast<uint32_t*>(idx->excode);
            switch (EX) {
                case 2: transform_excode_kernel<2><<<2368, 256>>>(raw, dst, N, (int)D); break;
                case 3: transform_excode_kernel<3><<<2368, 256>>>(raw, dst, N, (int)D); break;
                case 4: transform_excode_kernel<4><<<2368, 256>>>(raw, dst, N, (int)D); break;
                case 6: transform_excode_kernel<6><<<2368, 256>>>(raw, dst, N, (int)D); break;
                case 7: transform_excode_kernel<7><<<2368, 256>>>(raw, dst, N, (int)D); break;
                default: transform_excode_kernel<8><<<2368, 256>>>(raw, dst, N, (int)D); break;
            }
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
            if (e != cudaSuccess)
                s = fail(ERQ_ERR_CUDA, "EX-code layout kernel failed: %s", cudaGetErrorString(e));
        }
        cudaFree(raw);
        if (s != ERQ_OK) return s;
    }
    ERQ_TRY(dev_alloc(idx, &idx->xipnorm, N));
    ERQ_TRY(read_to_device(f.get(), idx->xipnorm, N * sizeof(float), staging, "the EX factors"));
    ERQ_TRY(dev_alloc(idx, &idx->ids, N));
    ERQ_TRY(read_to_device(f.get(), idx->ids, N * sizeof(uint32_t), staging, "the ids"));
    ERQ_TRY(dev_alloc(idx, &idx->c_first_block, K));
    ERQ_TRY(dev_alloc(idx, &idx->c_first_vec, K));
    ERQ_TRY(dev_alloc(idx, &idx->c_size, K));
    ERQ_TRY(dev_alloc(idx, &idx->c_nblocks, K));
    ERQ_CUDA(cudaMemcpy(idx->c_first_block, first_block.data(), K * 4, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(idx->c_first_vec, first_vec.data(), K * 4, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(idx->c_size, csize.data(), K * 4, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(idx->c_nblocks, idx->h_nblocks.data(), K * 4, cudaMemcpyHostToDevice));
    {
        std::vector<uint32_t> byz(K), rank(K);
        std::iota(byz.begin(), byz.end(), 0u);
        std::stable_sort(byz.begin(), byz.end(),
                         [&](uint32_t x, uint32_t y) { return csize[x] > csize[y]; });
        for (uint64_t r = 0; r < K; ++r) rank[byz[r]] = (uint32_t)r;
        ERQ_TRY(dev_alloc(idx, &idx->c_size_rank, K));
        ERQ_CUDA(cudaMemcpy(idx->c_size_rank, rank.data(), K * 4, cudaMemcpyHostToDevice));
        ERQ_TRY(dev_alloc(idx, &idx->c_by_size, K));
        ERQ_CUDA(cudaMemcpy(idx->c_by_size, byz.data(), K * 4, cudaMemcpyHostToDevice));
    }
    // split-BF16 GEMM operands: centroids and the rows of P^T
    ERQ_TRY(dev_alloc(idx, &idx->c_split, K * 3 * D));
    ERQ_TRY(dev_alloc(idx, &idx->pt_split, D * 3 * D));
    ERQ_TRY(dev_alloc(idx, &idx->cn, K));
    ERQ_TRY(dev_alloc(idx, &idx->c_chain, K * D));
    {
        std::vector<float> hp(D * D), hpt(D * D);
        ERQ_CUDA(cudaMemcpy(hp.data(), idx->P, D * D * 4, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < D; ++i)
            for (uint64_t j = 0; j < D; ++j) hpt[j * D + i] = hp[i * D + j];
        float* tmp = nullptr;
        ERQ_CUDA(cudaMalloc(&tmp, D * D * 4));
        cudaError_t e = cudaMemcpy(tmp, hpt.data(), D * D * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            split_rows_kernel<<<(unsigned)D, 256>>>(tmp, (int)D, (int)D, (int)D, false,
                                                    idx->pt_split, nullptr);
            split_rows_kernel<<<(unsigned)K, 256>>>(idx->centroids, (int)K, (int)D, (int)D, false,
                                                    idx->c_split, idx->cn);
            chain_layout_kernel<<<1184, 256>>>(idx->centroids, (int)K, (int)D, idx->c_chain);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
        }
        cudaFree(tmp);
        if (e != cudaSuccess) return fail(ERQ_ERR_CUDA, "split operands: %s", cudaGetErrorString(e));
        std::vector<float> hcn(K);
        ERQ_CUDA(cudaMemcpy(hcn.data(), idx->cn, K * 4, cudaMemcpyDeviceToHost));
        idx->cn_max = *std::max_element(hcn.begin(), hcn.end());
        // |estimate - true| <= (qn + cn) * (7 D u + 3.2 * 2^-16 + 3u) for the
        // split-BF16 products accumulated in FP32 plus the norm sums and the
        // epilogue; the reference's own L2Sqr16 value is within
        // 2 (D/16 + 6) u (qn + cn) of the true distance.  25% margin.
        const double u = std::ldexp(1.0, -24);
        const double dd = (double)D;
        idx->eps_rel = (float)(1.25 * (7 * dd * u + 3.2 * std::ldexp(1.0, -16) + 3 * u +
                                       2 * (dd / 16 + 6) * u));
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = idx->device;
    ERQ_CUDA(cudaMemPoolCreate(&idx->pool, &props));
    uint64_t keep = ~0ull;
    ERQ_CUDA(cudaMemPoolSetAttribute(idx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    return ERQ_OK;
}

// ------------------------------------------------------------ pipeline
size_t refine_smem_bytes(int D, int k, bool wide = false) {
    const int kpad = (k + 31) & ~31;
    return refine_smem_bytes_per_query(D, kpad, wide ? kWideWindowBlocks : kWindowBlocks);
}

// Streaming multiprocessors of the current device (cached per device).
int device_sms() {
    static int sms[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!sms[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        sms[dev] = n;
    }
    return sms[dev];
}

// The limits cover the largest k, so a later call with a smaller k never
// lowers them below what a captured graph's launches need.
template <int EX>
erq_status configure_refine(int D) {
    ERQ_CUDA(cudaFuncSetAttribute(refine_kernel<EX, 4, kWindowBlocks>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)refine_smem_bytes(D, kMaxTopK)));
    ERQ_CUDA(cudaFuncSetAttribute(refine_kernel<EX, kWideWarps, kWideWindowBlocks>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)refine_smem_bytes(D, kMaxTopK, true)));
    return ERQ_OK;
}
int next_pow2(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

erq_status configure_kernels(int D, int K, int k) {
    const int kp2 = next_pow2(K);

    ERQ_CUDA(cudaFuncSetAttribute(scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)scan_smem_bytes(D)));
    ERQ_CUDA(cudaFuncSetAttribute(probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)probe_smem_bytes(D, std::min(kp2, kProbeSortSmemKeys),
                                                        K <= kProbeStageKeys ? K : 0)));
    ERQ_CUDA(cudaFuncSetAttribute(probe_exact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)probe_exact_smem_bytes(D, std::min(kp2, kProbeSortSmemKeys))));
    for (const void* f : {(const void*)probe_warp_kernel<0>, (const void*)probe_warp_kernel<1>,
                          (const void*)probe_warp_kernel<2>})
        ERQ_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(kProbeWarpWarps * probe_warp_smem_per_warp(D))));
    ERQ_CUDA(cudaFuncSetAttribute(scan_lowacc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)low_scan_smem_bytes(D)));
    {
        const int smem = (int)(kLowRefineWarps * low_refine_smem_per_warp(D, kMaxTopK));
        ERQ_CUDA(cudaFuncSetAttribute(refine_lowacc_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ERQ_CUDA(cudaFuncSetAttribute(refine_lowacc_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ERQ_CUDA(cudaFuncSetAttribute(refine_lowacc_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ERQ_CUDA(cudaFuncSetAttribute(refine_lowacc_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ERQ_CUDA(cudaFuncSetAttribute(refine_lowacc_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        ERQ_CUDA(cudaFuncSetAttribute(refine_lowacc_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    }
    ERQ_TRY(configure_refine<2>(D));
    ERQ_TRY(configure_refine<3>(D));
    ERQ_TRY(configure_refine<4>(D));
    ERQ_TRY(configure_refine<6>(D));
    ERQ_TRY(configure_refine<7>(D));
    ERQ_TRY(configure_refine<8>(D));
    return ERQ_OK;
}

// ------------------------------------------------------------ tcgen05 GEMM
constexpr int kMaxDevices = 64;
// Wait status of gemm_tc_kernel (bit 0: a bounded wait ran out), one word per
// device image of the library.
__device__ uint32_t g_tc_status;

erq_status tc_status_ptr(uint32_t** out) {
    static std::mutex mu;
    static uint32_t* ptrs[kMaxDevices] = {};
    int dev = 0;
    ERQ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(ERQ_ERR_UNSUPPORTED, "device ordinal %d", dev);
    std::lock_guard<std::mutex> g(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        ERQ_CUDA(cudaGetSymbolAddress(&p, g_tc_status));
        ptrs[dev] = static_cast<uint32_t*>(p);
    }
    *out = ptrs[dev];
    return ERQ_OK;
}

// Copies the status word into pinned host memory on `st` (before a call
// synchronises); tc_status_check reads it afterwards.
erq_status tc_status_fetch(cudaStream_t st, uint32_t** host_word) {
    static std::mutex mu;
    static uint32_t* pinned[kMaxDevices] = {};
    uint32_t* dword = nullptr;
    ERQ_TRY(tc_status_ptr(&dword));
    int dev = 0;
    ERQ_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> g(mu);
        if (!pinned[dev]) {
            ERQ_CUDA(cudaMallocHost(&pinned[dev], sizeof(uint32_t)));
            *pinned[dev] = 0;
        }
    }
    ERQ_CUDA(cudaMemcpyAsync(pinned[dev], dword, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    *host_word = pinned[dev];
    return ERQ_OK;
}
// The status word read now (the caller has synchronised its work).
erq_status tc_status_check_now() {
    uint32_t* dword = nullptr;
    ERQ_TRY(tc_status_ptr(&dword));
    uint32_t v = 0;
    ERQ_CUDA(cudaMemcpy(&v, dword, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (v) {
        ERQ_CUDA(cudaMemset(dword, 0, sizeof(uint32_t)));
        return fail(ERQ_ERR_TIMEOUT, "a bounded wait in a kernel ran out; results are incomplete");
    }
    return ERQ_OK;
}

erq_status tc_status_check(uint32_t* host_word) {
    if (host_word && *host_word) {
        *host_word = 0;
        uint32_t* dword = nullptr;
        ERQ_TRY(tc_status_ptr(&dword));
        ERQ_CUDA(cudaMemset(dword, 0, sizeof(uint32_t)));
        return fail(ERQ_ERR_TIMEOUT, "a bounded wait in a kernel (tcgen05 GEMM or staged scan) ran out; results are incomplete");
    }
    return ERQ_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    });
    return fn;
}

// 2-D map of a row-major BF16 matrix [rows][cols]: boxes of 64 columns
// (128 bytes, the swizzle span) by box_rows rows, 128-byte swizzle, zero fill
// outside the matrix.
erq_status tensor_map_bf16(CUtensorMap* m, const void* ptr, uint64_t rows, uint64_t cols,
                           uint32_t box_rows) {
    auto fn = tensor_map_encoder();
    if (!fn) return fail(ERQ_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    if ((reinterpret_cast<uintptr_t>(ptr) & 15) || (cols * 2) % 16)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "TMA operand not 16-byte aligned");
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {cols * 2};
    cuuint32_t box[2] = {64, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(ERQ_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return ERQ_OK;
}

// C[M][N] = A[M][Kd] * B[N][Kd]^T (BF16, FP32 accumulate) with an epilogue,
// on tcgen05 (gemm_tc.cuh).  Kd must be a multiple of 64.
// Polls per pipeline wait of the tcgen05 GEMM; lowered only by
// erq_debug_set_gemm_wait_limit to exercise the timeout path.
std::atomic<uint32_t> g_tc_wait_limit{kTcWaitLimit};

erq_status gemm_tc(const __nv_bfloat16* A, const __nv_bfloat16* B, float* C, int M, int N, int Kd,
                   const GemmEpilogue& epi, int kernel_id, cudaStream_t st) {
    if (M <= 0 || N <= 0) return ERQ_OK;
    if (Kd <= 0 || Kd % kTcBK) return fail(ERQ_ERR_INVALID_ARGUMENT, "GEMM depth %d not a multiple of 64", Kd);
    CUtensorMap ta, tb;
    ERQ_TRY(tensor_map_bf16(&ta, A, (uint64_t)M, (uint64_t)Kd, kTcBM));
    ERQ_TRY(tensor_map_bf16(&tb, B, (uint64_t)N, (uint64_t)Kd, kTcBN));
    uint32_t* status = nullptr;
    ERQ_TRY(tc_status_ptr(&status));
    {
        static std::mutex mu;
        static bool configured[kMaxDevices] = {};
        int dev = 0;
        ERQ_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> g(mu);
        if (!configured[dev]) {
            ERQ_CUDA(cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)gemm_tc_smem_bytes()));
            configured[dev] = true;
        }
    }
    // persistent: one CTA per SM (the ring leaves room for one), at most one per tile
    const uint64_t tiles = (uint64_t)div_up(N, kTcBN) * (uint64_t)div_up(M, kTcBM);
    if (tiles > 0x7fffffffull) return fail(ERQ_ERR_INVALID_ARGUMENT, "GEMM of %llu tiles", (unsigned long long)tiles);
    const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)device_sms());
    LaunchTimer t(kernel_id, st);
    gemm_tc_kernel<<<grid, kTcThreads, gemm_tc_smem_bytes(), st>>>(ta, tb, C, M, N, Kd, epi, status,
                                                                    g_tc_wait_limit.load());
    t.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

// Device buffers of one query batch.
struct Batch {
    const float* qrot = nullptr;  // [nq][D] on device
    uint64_t nq = 0;
    float* dist = nullptr;        // [nq][K]
    uint32_t* probe_cid = nullptr;
    float* probe_sqy = nullptr;
    uint64_t* s_off = nullptr;
    int32_t* S = nullptr;
    float* delta = nullptr;
    float* sumq = nullptr;
    float* vl = nullptr;              // [nq][nprobe] lower query range end (4-factor format)
    __nv_bfloat16* qsplit = nullptr;  // [nq][3D] split rotated queries
    float* qn = nullptr;              // [nq]
    // work order (order.cuh)
    uint32_t* keys = nullptr;         // [nq * nprobe]
    uint32_t* keys_q = nullptr;       // [nq]
    uint32_t* buckets = nullptr;      // [K + 1] pair sort; ends of each cluster's run after it
    uint32_t* buckets_q = nullptr;    // [K + 1] query sort, right after buckets
    uint32_t* order_pairs = nullptr;  // [nq * nprobe]
    uint32_t* order_q = nullptr;      // [nq]
    float* bmin = nullptr;            // smallest lower bound per scanned block (S / 32 entries)
    uint32_t* fb_flag = nullptr;      // [nq] queries whose probe needs all K exact distances
    uint64_t* sortbuf = nullptr;      // [nq][sort_cap] probe sort keys too many for shared memory
    uint64_t sort_cap = 0;
    // a split probe's sorted lists (launch_probe_tc / launch_probe_finish);
    // allocated by the learned paths only
    uint64_t* plist = nullptr;        // [nq][kProbeWarpCap]
    uint32_t* plist_n = nullptr;      // [nq]
    uint64_t* plist_cut = nullptr;    // [nq]
};

template <class Alloc>
erq_status alloc_probe_lists(Alloc& s, uint64_t nq, Batch& b) {
    ERQ_TRY(s.alloc(&b.plist, nq * kProbeWarpCap));
    ERQ_TRY(s.alloc(&b.plist_n, nq));
    ERQ_TRY(s.alloc(&b.plist_cut, nq));
    return ERQ_OK;
}

int probe_candidates(uint64_t nprobe);

// Sort keys per query the probe kernels keep in global memory (0: all fit in
// shared memory): the selection of probe_kernel (Msel candidates, with the 64
// feature ranks when `features`) and the nprobe slots of probe_exact_kernel.
uint64_t probe_sort_cap(const erq_index* idx, uint64_t nprobe, bool features) {
    const int K = (int)idx->K;
    const int n = (int)std::min<uint64_t>(nprobe, idx->K);
    const int msel = features ? std::max(probe_candidates(n), kProbeFeatRank) : probe_candidates(n);
    const int spow2 = next_pow2(msel + 1 > K ? K : msel);
    const int npow2 = next_pow2(n);
    const int cap = std::max(spow2, npow2);
    return cap > kProbeSortSmemKeys ? (uint64_t)cap : 0;
}

// Largest query batch whose scan workspace fits the budget.
uint64_t batch_queries(const erq_index* idx, uint64_t nprobe, uint64_t nq) {
    const uint64_t per_q = 32ull * idx->top_blocks[nprobe] * sizeof(int32_t) +
                           idx->K * sizeof(float) + nprobe * 28 + 6 * idx->D + 4 +
                           idx->top_blocks[nprobe] * sizeof(float);
    const uint64_t per_q_all = per_q + probe_sort_cap(idx, nprobe, true) * sizeof(uint64_t);
    const uint64_t budget = 3ull << 30;
    uint64_t b = std::max<uint64_t>(1, budget / std::max<uint64_t>(per_q_all, 1));
    return std::min(b, nq);
}

template <class Alloc>
erq_status alloc_batch(Alloc& s, const erq_index* idx, uint64_t nq, uint64_t nprobe, Batch& b) {
    b.nq = nq;
    ERQ_TRY(s.alloc(&b.dist, nq * idx->K));
    ERQ_TRY(s.alloc(&b.probe_cid, nq * nprobe));
    ERQ_TRY(s.alloc(&b.probe_sqy, nq * nprobe));
    ERQ_TRY(s.alloc(&b.s_off, nq * nprobe));
    ERQ_TRY(s.alloc(&b.S, nq * 32ull * idx->top_blocks[nprobe]));
    ERQ_TRY(s.alloc(&b.delta, nq * nprobe));
    ERQ_TRY(s.alloc(&b.sumq, nq * nprobe));
    ERQ_TRY(s.alloc(&b.vl, nq * nprobe));
    ERQ_TRY(s.alloc(&b.qsplit, nq * 3 * idx->D));
    ERQ_TRY(s.alloc(&b.qn, nq));
    ERQ_TRY(s.alloc(&b.keys, nq * nprobe));
    ERQ_TRY(s.alloc(&b.keys_q, nq));
    ERQ_TRY(s.alloc(&b.buckets, 2 * (idx->K + 1)));
    b.buckets_q = b.buckets + idx->K + 1;
    ERQ_TRY(s.alloc(&b.order_pairs, nq * nprobe));
    ERQ_TRY(s.alloc(&b.order_q, nq));
    ERQ_TRY(s.alloc(&b.bmin, nq * idx->top_blocks[nprobe]));
    ERQ_TRY(s.alloc(&b.fb_flag, nq));
    b.sort_cap = probe_sort_cap(idx, nprobe, true);
    if (b.sort_cap) ERQ_TRY(s.alloc(&b.sortbuf, nq * b.sort_cap));
    return ERQ_OK;
}

// Both work orders at once: (query, probe) pairs by cluster id (or by the
// cluster's size rank) into b.order_pairs, runs delimited by b.buckets (pairs
// a per-query probe count leaves out go last), and queries by the size rank
// of their nearest cluster into b.order_q.  One memset and three kernels.
erq_status order_both(const erq_index* idx, const Batch& b, uint64_t nprobe, cudaStream_t st,
                      const int* q_nprobe, bool pairs_by_size) {
    const uint64_t pairs = b.nq * nprobe;
    const uint32_t nb = (uint32_t)idx->K + 1;
    ERQ_CUDA(cudaMemsetAsync(b.buckets, 0, 2ull * nb * sizeof(uint32_t), st));
    if (pairs == 0) return ERQ_OK;
    const unsigned grid = (unsigned)div_up(pairs, 256);
    {
        LaunchTimer t(kOrder, st);
        order_keys_count_kernel<<<grid, 256, 0, st>>>(
            b.probe_cid, (uint32_t)pairs, (uint32_t)b.nq, (int)nprobe, q_nprobe, (uint32_t)idx->K,
            pairs_by_size, idx->c_size_rank, b.keys, b.buckets, b.keys_q, b.buckets_q);
        t.finish();
    }
    {
        LaunchTimer t(kOrder, st);
        bucket_scan_kernel<<<2, kBucketScanThreads, 0, st>>>(b.buckets, b.buckets_q, nb);
        t.finish();
    }
    {
        LaunchTimer t(kOrder, st);
        bucket_scatter2_kernel<<<grid, 256, 0, st>>>(b.keys, (uint32_t)pairs, b.buckets, b.order_pairs,
                                                     b.keys_q, (uint32_t)b.nq, b.buckets_q, b.order_q);
        t.finish();
    }
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

// Both orders for the per-pair scan and the refinement.  Small batches gain
// nothing from reuse and keep the identity order (returns false).
bool launch_order(const erq_index* idx, const Batch& b, uint64_t nprobe, cudaStream_t st,
                  const int* q_nprobe, erq_status* err) {
    *err = ERQ_OK;
    if (b.nq * nprobe < 1024 || !b.order_pairs) return false;
    if ((*err = order_both(idx, b, nprobe, st, q_nprobe, true)) != ERQ_OK) return false;
    return true;
}

// Candidate count for the probe: nprobe plus a margin (probe.cuh).  When the
// margin does not prove the cut the kernel computes all K exact distances
// (counted in g_probe_fallbacks).
int probe_candidates(uint64_t nprobe) {
    return (int)(nprobe + std::max<uint64_t>(32, nprobe / 2));
}

// Queries whose probe fell back to all K exact distances, per device image.
__device__ uint32_t g_probe_fallbacks;
uint32_t* probe_fallback_counter() {
    static uint32_t* ptrs[kMaxDevices] = {};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_probe_fallbacks) != cudaSuccess) return nullptr;
        ptrs[dev] = static_cast<uint32_t*>(p);
    }
    return ptrs[dev];
}

// Refinement statistics (RefineArgs::stats), per device image, counted while
// g_refine_stats_on is set (erq_debug_refine_stats).
__device__ unsigned long long g_refine_stats[4];
std::atomic<bool> g_refine_stats_on{false};
unsigned long long* refine_stats_counter() {
    static unsigned long long* ptrs[kMaxDevices] = {};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> g(mu);
    if (!ptrs[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_refine_stats) != cudaSuccess) return nullptr;
        ptrs[dev] = static_cast<unsigned long long*>(p);
    }
    return ptrs[dev];
}

// Coarse probe on tensor cores: split the rotated queries, estimate all
// distances with the split-BF16 GEMM, then the exact probe kernel.
// The arguments of the probe kernels for a batch (near_d: the features' 64
// smallest estimates are wanted).
erq_status probe_args(const erq_index* idx, const Batch& b, uint64_t nprobe, float* near_d,
                      ProbeArgs& a, int& npow2) {
    const int D = (int)idx->D, K = (int)idx->K;
    a = ProbeArgs{};
    a.approx = b.dist;
    a.qrot = b.qrot;
    a.centroids = idx->c_chain;
    a.qn = b.qn;
    a.c_nblocks = idx->c_nblocks;
    a.cn_max = idx->cn_max;
    a.eps_rel = idx->eps_rel;
    a.stride = 32ull * idx->top_blocks[nprobe];
    a.probe_cid = b.probe_cid;
    a.probe_sqy = b.probe_sqy;
    a.s_off = b.s_off;
    a.fallbacks = probe_fallback_counter();
    a.near_d = near_d;
    a.nq = (int)b.nq;
    a.K = K;
    a.Kpow2 = next_pow2(K);
    a.D = D;
    a.nprobe = (int)nprobe;
    a.check_rank = (int)nprobe;
    a.M = probe_candidates(a.check_rank);
    {
        const int msel = near_d ? std::max(a.M, kProbeFeatRank) : a.M;
        a.Spow2 = next_pow2(msel + 1 > K ? K : msel);
    }
    if (!b.fb_flag) return fail(ERQ_ERR_INVALID_ARGUMENT, "probe batch without fallback flags");
    a.fallback_flag = b.fb_flag;
    a.stage_keys = K <= kProbeStageKeys ? 1 : 0;
    a.exact_rows = b.dist;
    a.list = b.plist;
    a.list_n = b.plist_n;
    a.list_cut = b.plist_cut;
    npow2 = next_pow2((int)std::min<uint64_t>(nprobe, (uint64_t)K));
    if (a.Spow2 > kProbeSortSmemKeys || npow2 > kProbeSortSmemKeys) {
        if (!b.sortbuf || b.sort_cap < (uint64_t)std::max(a.Spow2, npow2))
            return fail(ERQ_ERR_INVALID_ARGUMENT, "probe batch without a large enough sort buffer");
        a.sort_global = b.sortbuf;
        a.sort_cap = b.sort_cap;
    }
    return ERQ_OK;
}

// a warp per query when the candidate list fits its registers
bool probe_warp_form(const ProbeArgs& a) {
    const int msel = a.near_d ? std::max(a.M, kProbeFeatRank) : a.M;
    return !a.sort_global && a.K > kProbeWarpCap && msel < kProbeWarpCap;
}

// The fallback of the probe kernels: all K exact distances for the queries
// whose cut was not proven.
erq_status launch_probe_exact(const Batch& b, const ProbeArgs& a, int npow2, cudaStream_t st) {
    LaunchTimer t(kProbe, st);
    probe_exact_kernel<<<(unsigned)b.nq, kProbeThreads,
                         probe_exact_smem_bytes(a.D, a.sort_global ? 0 : npow2), st>>>(a, 1, npow2);
    t.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

// The coarse probe of a batch: split + estimate GEMM + exact top nprobe.
// With `split` (and the batch's probe lists), a probe that runs in the warp
// form stops after the features and the sorted lists (*split set): the rest
// follows in launch_probe_finish once each query's depth is known.
erq_status launch_probe_tc(const erq_index* idx, const Batch& b, uint64_t nprobe, cudaStream_t st,
                           float* near_d = nullptr, bool* split = nullptr) {
    const int D = (int)idx->D, K = (int)idx->K;
    if (split) *split = false;
    {
        LaunchTimer t(kSplit, st);
        split_rows_kernel<<<(unsigned)b.nq, 256, 0, st>>>(b.qrot, (int)b.nq, D, D, true, b.qsplit,
                                                          b.qn);
        t.finish();
        ERQ_CUDA(cudaGetLastError());
    }
    {
        GemmEpilogue epi;
        epi.row_norm = b.qn;
        epi.col_norm = idx->cn;
        ERQ_TRY(gemm_tc(b.qsplit, idx->c_split, b.dist, (int)b.nq, K, 3 * D, epi, kGemm, st));
    }
    ProbeArgs a;
    int npow2 = 0;
    ERQ_TRY(probe_args(idx, b, nprobe, near_d, a, npow2));
    const bool warp_form = probe_warp_form(a);
    const bool first_of_two = warp_form && split && b.plist;
    {
        LaunchTimer t(kProbe, st);
        const unsigned wgrid = (unsigned)div_up(b.nq, kProbeWarpWarps);
        const size_t wsmem = kProbeWarpWarps * probe_warp_smem_per_warp(D);
        if (first_of_two)
            probe_warp_kernel<1><<<wgrid, kProbeWarpWarps * 32, wsmem, st>>>(a);
        else if (warp_form)
            probe_warp_kernel<0><<<wgrid, kProbeWarpWarps * 32, wsmem, st>>>(a);
        else
            probe_kernel<<<(unsigned)b.nq, kProbeThreads,
                           probe_smem_bytes(D, a.sort_global ? 0 : a.Spow2, a.stage_keys ? K : 0), st>>>(a);
        t.finish();
        ERQ_CUDA(cudaGetLastError());
    }
    if (first_of_two) {
        *split = true;
        return ERQ_OK;
    }
    return launch_probe_exact(b, a, npow2, st);
}

// The second launch of a split probe: each query's exact distances up to the
// depth q_check[q] it will scan (at most nprobe), from its sorted list.
erq_status launch_probe_finish(const erq_index* idx, const Batch& b, uint64_t nprobe, cudaStream_t st,
                               const int* q_check) {
    ProbeArgs a;
    int npow2 = 0;
    ERQ_TRY(probe_args(idx, b, nprobe, nullptr, a, npow2));
    a.q_check = q_check;
    {
        LaunchTimer t(kProbe, st);
        probe_warp_kernel<2><<<(unsigned)div_up(b.nq, kProbeWarpWarps), kProbeWarpWarps * 32,
                               kProbeWarpWarps * probe_warp_smem_per_warp(a.D), st>>>(a);
        t.finish();
        ERQ_CUDA(cudaGetLastError());
    }
    return launch_probe_exact(b, a, npow2, st);
}

erq_status launch_probe(const erq_index* idx, const Batch& b, uint64_t nprobe, cudaStream_t st) {
    const int D = (int)idx->D, K = (int)idx->K;
    dim3 g1((unsigned)div_up(K, kCdTC), (unsigned)div_up(b.nq, kCdTQ));
    LaunchTimer t1(kCentroidDist, st);
    centroid_dist_kernel<<<g1, 256, 0, st>>>(b.qrot, (int)b.nq, idx->centroids, K, D, b.dist);
    t1.finish();
    ERQ_CUDA(cudaGetLastError());
    ProbeArgs a{};
    a.qrot = b.qrot;
    a.centroids = idx->c_chain;  // unused: the rows already hold exact distances
    a.c_nblocks = idx->c_nblocks;
    a.stride = 32ull * idx->top_blocks[nprobe];
    a.probe_cid = b.probe_cid;
    a.probe_sqy = b.probe_sqy;
    a.s_off = b.s_off;
    a.nq = (int)b.nq;
    a.K = K;
    a.Kpow2 = next_pow2(K);
    a.D = D;
    a.nprobe = (int)nprobe;
    a.exact_rows = b.dist;
    const int npow2 = next_pow2((int)std::min<uint64_t>(nprobe, (uint64_t)K));
    if (npow2 > kProbeSortSmemKeys) {
        if (!b.sortbuf || b.sort_cap < (uint64_t)npow2)
            return fail(ERQ_ERR_INVALID_ARGUMENT, "probe batch without a large enough sort buffer");
        a.sort_global = b.sortbuf;
        a.sort_cap = b.sort_cap;
    }
    LaunchTimer t2(kSelectProbe, st);
    probe_exact_kernel<<<(unsigned)b.nq, kProbeThreads, probe_exact_smem_bytes(D, a.sort_global ? 0 : npow2),
                         st>>>(a, 0, npow2);
    t2.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

LowFactors low_factors(const erq_index* idx) {
    LowFactors f;
    f.x2 = idx->onorm;
    f.fip = idx->fac_ip;
    f.sumxb = idx->fac_sumxb;
    f.ferr = idx->fac_err;
    return f;
}

// The scan of the 4-factor format (lowacc.cuh): width, vl and sum(q - c)/2
// land in b.delta, b.vl and b.sumq.
erq_status launch_scan_lowacc(const erq_index* idx, const Batch& b, uint64_t nprobe, cudaStream_t st) {
    LowScanArgs a{};
    a.qrot = b.qrot;
    a.centroids = idx->centroids;
    a.probe_cid = b.probe_cid;
    a.probe_sqy = b.probe_sqy;
    a.codes = idx->codes;
    a.c_first_block = idx->c_first_block;
    a.c_nblocks = idx->c_nblocks;
    a.c_size = idx->c_size;
    a.s_off = b.s_off;
    a.S = b.S;
    a.qp_width = b.delta;
    a.qp_vl = b.vl;
    a.qp_half = b.sumq;
    a.bmin = b.bmin;
    a.f = low_factors(idx);
    a.D = (int)idx->D;
    a.nprobe = (int)nprobe;
    ERQ_TRY(tc_status_ptr(&a.status));
    const uint64_t pairs = b.nq * nprobe;
    if (pairs > 0x7fffffffull) return fail(ERQ_ERR_INVALID_ARGUMENT, "too many (query, probe) pairs");
    LaunchTimer t(kScan, st);
    scan_lowacc_kernel<<<(unsigned)pairs, kScanWarps * 32, low_scan_smem_bytes(a.D), st>>>(a);
    t.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

erq_status launch_scan(const erq_index* idx, const Batch& b, uint64_t nprobe, cudaStream_t st,
                       const int* q_nprobe = nullptr, const uint32_t* order = nullptr) {
    if (idx->factors == 4) {
        if (q_nprobe || order)
            return fail(ERQ_ERR_UNSUPPORTED, "per-query depths and work orders take one-factor indexes");
        return launch_scan_lowacc(idx, b, nprobe, st);
    }
    ScanArgs a{};
    a.order = order;
    a.onorm = idx->onorm;
    a.c_size = idx->c_size;
    a.bmin = b.bmin;
    a.qrot = b.qrot;
    a.centroids = idx->centroids;
    a.probe_cid = b.probe_cid;
    a.probe_sqy = b.probe_sqy;
    a.codes = idx->codes;
    a.c_first_block = idx->c_first_block;
    a.c_nblocks = idx->c_nblocks;
    a.s_off = b.s_off;
    a.S = b.S;
    a.qp_delta = b.delta;
    a.qp_sumq = b.sumq;
    a.q_nprobe = q_nprobe;
    a.D = (int)idx->D;
    a.nprobe = (int)nprobe;
    ERQ_TRY(tc_status_ptr(&a.status));
    const uint64_t pairs = b.nq * nprobe;
    if (pairs > 0x7fffffffull) return fail(ERQ_ERR_INVALID_ARGUMENT, "too many (query, probe) pairs");
    LaunchTimer t(kScan, st);
    scan_kernel<<<(unsigned)pairs, kScanWarps * 32, scan_smem_bytes(a.D), st>>>(a);
    t.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

// refine_warps: 4 or kWideWarps chooses the form; 0 takes the wide one when
// the batch has no more queries than SMs.
erq_status launch_refine(const erq_index* idx, const Batch& b, uint64_t nprobe, uint64_t k,
                         uint32_t* out_ids, float* out_dists, cudaStream_t st,
                         const int* q_nprobe = nullptr, const uint32_t* order = nullptr,
                         int refine_warps = 0) {
    if (idx->factors == 4) {
        if (q_nprobe || order)
            return fail(ERQ_ERR_UNSUPPORTED, "per-query depths and work orders take one-factor indexes");
        LowRefineArgs a{};
        a.qrot = b.qrot;
        a.centroids = idx->centroids;
        a.probe_cid = b.probe_cid;
        a.probe_sqy = b.probe_sqy;
        a.s_off = b.s_off;
        a.S = b.S;
        a.qp_width = b.delta;
        a.qp_vl = b.vl;
        a.qp_half = b.sumq;
        a.bmin = b.bmin;
        a.f = low_factors(idx);
        a.excode = idx->excode;
        a.ex_row = idx->ex_row;
        a.xipnorm = idx->xipnorm;
        a.ids = idx->ids;
        a.c_first_block = idx->c_first_block;
        a.c_first_vec = idx->c_first_vec;
        a.c_size = idx->c_size;
        a.out_ids = out_ids;
        a.out_dists = out_dists;
        a.nq = (int)b.nq;
        a.D = (int)idx->D;
        a.EX = (int)idx->EX;
        a.nprobe = (int)nprobe;
        a.k = (int)k;
        const unsigned grid = (unsigned)div_up(b.nq, kLowRefineWarps);
        const size_t smem = kLowRefineWarps * low_refine_smem_per_warp(a.D, (a.k + 31) & ~31);
        LaunchTimer t(kRefine, st);
        switch (idx->EX) {
            case 2: refine_lowacc_kernel<2><<<grid, kLowRefineWarps * 32, smem, st>>>(a); break;
            case 3: refine_lowacc_kernel<3><<<grid, kLowRefineWarps * 32, smem, st>>>(a); break;
            case 4: refine_lowacc_kernel<4><<<grid, kLowRefineWarps * 32, smem, st>>>(a); break;
            case 6: refine_lowacc_kernel<6><<<grid, kLowRefineWarps * 32, smem, st>>>(a); break;
            case 7: refine_lowacc_kernel<7><<<grid, kLowRefineWarps * 32, smem, st>>>(a); break;
            case 8: refine_lowacc_kernel<8><<<grid, kLowRefineWarps * 32, smem, st>>>(a); break;
            default: return fail(ERQ_ERR_FORMAT, "bad EX");
        }
        t.finish();
        ERQ_CUDA(cudaGetLastError());
        return ERQ_OK;
    }
    RefineArgs a{};
    a.order = order;
    a.bmin = b.bmin;
    a.stats = g_refine_stats_on.load() ? refine_stats_counter() : nullptr;
    a.qrot = b.qrot;
    a.centroids = idx->centroids;
    a.probe_cid = b.probe_cid;
    a.probe_sqy = b.probe_sqy;
    a.s_off = b.s_off;
    a.S = b.S;
    a.qp_delta = b.delta;
    a.qp_sumq = b.sumq;
    a.onorm = idx->onorm;
    a.excode = idx->excode;
    a.ex_row = idx->ex_row;
    a.xipnorm = idx->xipnorm;
    a.ids = idx->ids;
    a.c_first_block = idx->c_first_block;
    a.c_first_vec = idx->c_first_vec;
    a.c_size = idx->c_size;
    a.out_ids = out_ids;
    a.out_dists = out_dists;
    a.q_nprobe = q_nprobe;
    a.nq = (int)b.nq;
    a.D = (int)idx->D;
    a.EX = (int)idx->EX;
    a.nprobe = (int)nprobe;
    a.k = (int)k;
    const unsigned grid = (unsigned)b.nq;
    const bool wide = refine_warps ? refine_warps == kWideWarps : b.nq <= (uint64_t)device_sms();
    const size_t smem = refine_smem_bytes(a.D, a.k, wide);
    LaunchTimer t(kRefine, st);
#define ERQ_REFINE_CASE(X)                                                                          \
    case X:                                                                                         \
        if (wide)                                                                                   \
            refine_kernel<X, kWideWarps, kWideWindowBlocks><<<grid, kWideWarps * 32, smem, st>>>(a); \
        else                                                                                        \
            refine_kernel<X, 4, kWindowBlocks><<<grid, kRefineThreads, smem, st>>>(a);              \
        break;
    switch (idx->EX) {
        ERQ_REFINE_CASE(2)
        ERQ_REFINE_CASE(3)
        ERQ_REFINE_CASE(4)
        ERQ_REFINE_CASE(6)
        ERQ_REFINE_CASE(7)
        ERQ_REFINE_CASE(8)
        default: return fail(ERQ_ERR_FORMAT, "bad EX");
    }
#undef ERQ_REFINE_CASE
    t.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

erq_status check_search_args(const erq_index* idx, uint64_t nq, uint64_t k, uint64_t nprobe,
                             const void* q, const void* ids) {
    if (!idx) return fail(ERQ_ERR_INVALID_ARGUMENT, "index is NULL");
    if (nq == 0) return ERQ_OK;
    if (!q || !ids) return fail(ERQ_ERR_INVALID_ARGUMENT, "queries and ids must not be NULL");
    if (k < 1 || k > (uint64_t)kMaxTopK)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "k=%llu outside [1, %d]", (unsigned long long)k, kMaxTopK);
    if (nprobe < 1 || nprobe > idx->K)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "nprobe=%llu outside [1, K=%llu]",
                    (unsigned long long)nprobe, (unsigned long long)idx->K);
    if (nq > (1ull << 30)) return fail(ERQ_ERR_INVALID_ARGUMENT, "nq too large");
    return ERQ_OK;
}

// Rotated queries on the device -> ids/dists on the device.
erq_status search_device(const erq_index* idx, const float* qrot_dev, uint64_t nq, uint64_t k,
                         uint64_t nprobe, uint32_t* ids_dev, float* dists_dev, cudaStream_t st) {
    ERQ_TRY(configure_kernels((int)idx->D, (int)idx->K, (int)k));
    const uint64_t bq = batch_queries(idx, nprobe, nq);
    Scratch s(st, idx->pool);
    Batch b;
    ERQ_TRY(alloc_batch(s, idx, bq, nprobe, b));
    for (uint64_t q0 = 0; q0 < nq; q0 += bq) {
        b.nq = std::min(bq, nq - q0);
        b.qrot = qrot_dev + q0 * idx->D;
        ERQ_TRY(launch_probe_tc(idx, b, nprobe, st));
        erq_status oe;
        const bool ordered = launch_order(idx, b, nprobe, st, nullptr, &oe);
        ERQ_TRY(oe);
        ERQ_TRY(launch_scan(idx, b, nprobe, st, nullptr, ordered ? b.order_pairs : nullptr));
        ERQ_TRY(launch_refine(idx, b, nprobe, k, ids_dev + q0 * k,
                              dists_dev ? dists_dev + q0 * k : nullptr, st, nullptr,
                              ordered ? b.order_q : nullptr));
    }
    return ERQ_OK;
}

// out[nq][D] = pad(q[nq][DIM]) * P on tensor cores (split-BF16, FP32 accumulation).
erq_status rotate_into(const erq_index* idx, const float* q_dev, uint64_t nq, float* out_dev,
                       __nv_bfloat16* qs, cudaStream_t st) {
    if (nq == 0) return ERQ_OK;
    const int D = (int)idx->D;
    {
        LaunchTimer t(kSplit, st);
        split_rows_kernel<<<(unsigned)nq, 256, 0, st>>>(q_dev, (int)nq, (int)idx->DIM, D, true, qs,
                                                        nullptr);
        t.finish();
        ERQ_CUDA(cudaGetLastError());
    }
    return gemm_tc(qs, idx->pt_split, out_dev, (int)nq, D, 3 * D, GemmEpilogue(), kRotate, st);
}

erq_status rotate_device(const erq_index* idx, const float* q_dev, uint64_t nq, float* out_dev,
                         cudaStream_t st) {
    if (nq == 0) return ERQ_OK;
    Scratch s(st, idx->pool);
    __nv_bfloat16* qs = nullptr;
    ERQ_TRY(s.alloc(&qs, nq * 3 * idx->D));
    return rotate_into(idx, q_dev, nq, out_dev, qs, st);
}

// Shared body of erq_search / erq_search_raw.
erq_status search_entry(const erq_index* idx, const float* queries, bool rotated, uint64_t nq,
                        uint64_t k, uint64_t nprobe, uint32_t* ids, float* dists, void* stream) {
    ERQ_TRY(check_search_args(idx, nq, k, nprobe, queries, ids));
    if (nq == 0) return ERQ_OK;
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint64_t in_cols = rotated ? idx->D : idx->DIM;
    const bool q_dev = is_device_ptr(queries);
    const bool ids_dev = is_device_ptr(ids);
    const bool d_dev = dists == nullptr || is_device_ptr(dists);
    if ((ids_dev && (reinterpret_cast<uintptr_t>(ids) & 3)) ||
        (dists && d_dev && (reinterpret_cast<uintptr_t>(dists) & 3)))
        return fail(ERQ_ERR_INVALID_ARGUMENT, "ids/dists device buffers must be 4-byte aligned");
    Scratch s(st, idx->pool);
    const float* qin = queries;
    // the kernels read queries as float4: device inputs off a 16-byte
    // boundary are copied into aligned scratch first
    if (!q_dev || (reinterpret_cast<uintptr_t>(queries) & 15)) {
        float* tmp = nullptr;
        ERQ_TRY(s.alloc(&tmp, nq * in_cols));
        ERQ_CUDA(cudaMemcpyAsync(tmp, queries, nq * in_cols * sizeof(float), cudaMemcpyDefault, st));
        qin = tmp;
    }
    const float* qrot = qin;
    if (!rotated) {
        float* tmp = nullptr;
        ERQ_TRY(s.alloc(&tmp, nq * idx->D));
        ERQ_TRY(rotate_device(idx, qin, nq, tmp, st));
        qrot = tmp;
    }
    uint32_t* ids_out = ids;
    float* d_out = dists;
    if (!ids_dev) ERQ_TRY(s.alloc(&ids_out, nq * k));
    if (!d_dev) ERQ_TRY(s.alloc(&d_out, nq * k));
    ERQ_TRY(search_device(idx, qrot, nq, k, nprobe, ids_out, d_out, st));
    const bool host_io = !q_dev || !ids_dev || !d_dev;
    if (!ids_dev)
        ERQ_CUDA(cudaMemcpyAsync(ids, ids_out, nq * k * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    if (!d_dev)
        ERQ_CUDA(cudaMemcpyAsync(dists, d_out, nq * k * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (host_io) {
        uint32_t* hw = nullptr;
        ERQ_TRY(tc_status_fetch(st, &hw));
        ERQ_CUDA(cudaStreamSynchronize(st));
        ERQ_TRY(tc_status_check(hw));
    }
    return ERQ_OK;
}

}  // namespace


// ----------------------------------------------------------- learned probing
struct erq_probe_model {
    int device = 0;
    float* w = nullptr;             // [kMlpParams] FP32 master weights
    __nv_bfloat16* wb = nullptr;    // [kMlpParams] BF16 copy used by the forward pass
    float* mean = nullptr;          // [kMlpIn] feature standardisation
    float* stdv = nullptr;          // [kMlpIn]
    int* bins_dev = nullptr;        // [kMlpBins] probe count of each class
    int bins[kMlpBins] = {};
    __nv_bfloat16* w1d = nullptr;   // [256][640] = [W1 | W1], tensor-core inference
    __nv_bfloat16* w2d = nullptr;   // [256][512] = [W2 | W2]

    ~erq_probe_model() {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        for (void* p : {(void*)w, (void*)wb, (void*)mean, (void*)stdv, (void*)bins_dev,
                        (void*)w1d, (void*)w2d})
            if (p) cudaFree(p);
        if (prev >= 0) cudaSetDevice(prev);
    }
};

namespace {

template <typename TB>
erq_status mlp_mm(const float* A, long sam, long sak, const TB* B, long sbk, long sbn, float* C,
                  int M, int N, int K, const float* bias, bool relu, cudaStream_t st) {
    dim3 grid((unsigned)div_up(N, 16), (unsigned)div_up(M, 16));
    LaunchTimer t(kMlp, st);
    mlp_matmul_kernel<TB><<<grid, 256, 0, st>>>(A, sam, sak, B, sbk, sbn, C, M, N, K, bias, relu,
                                                false);
    t.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

// Activations of one batch.
struct MlpWork {
    float* x = nullptr;   // [B][320] standardised features
    float* h1 = nullptr;  // [B][256]
    float* h2 = nullptr;  // [B][256]
    float* z = nullptr;   // [B][8]
    float* probs = nullptr;
    float* dz = nullptr;
    float* dh2 = nullptr;
    float* dh1 = nullptr;
    float* loss = nullptr;  // [B]
    __nv_bfloat16* xs = nullptr;  // [B][640] split inputs (inference)
    __nv_bfloat16* hs = nullptr;  // [B][512] split first hidden layer (inference)
};

template <class Alloc>
erq_status mlp_alloc(Alloc& s, int B, bool train, MlpWork& w) {
    ERQ_TRY(s.alloc(&w.x, (size_t)B * kMlpIn));
    ERQ_TRY(s.alloc(&w.h1, (size_t)B * kMlpHidden));
    ERQ_TRY(s.alloc(&w.h2, (size_t)B * kMlpHidden));
    ERQ_TRY(s.alloc(&w.z, (size_t)B * kMlpBins));
    ERQ_TRY(s.alloc(&w.probs, (size_t)B * kMlpBins));
    if (!train) {
        ERQ_TRY(s.alloc(&w.xs, (size_t)B * 2 * kMlpIn));
        ERQ_TRY(s.alloc(&w.hs, (size_t)B * 2 * kMlpHidden));
    }
    if (train) {
        ERQ_TRY(s.alloc(&w.dz, (size_t)B * kMlpBins));
        ERQ_TRY(s.alloc(&w.dh2, (size_t)B * kMlpHidden));
        ERQ_TRY(s.alloc(&w.dh1, (size_t)B * kMlpHidden));
        ERQ_TRY(s.alloc(&w.loss, (size_t)B));
    }
    return ERQ_OK;
}

// logits z = W3 relu(W2 relu(W1 x + b1) + b2) + b3, BF16 weights, FP32 sums.
erq_status mlp_forward(const erq_probe_model* m, const MlpWork& w, int B, cudaStream_t st) {
    ERQ_TRY(mlp_mm(w.x, kMlpIn, 1, m->wb + kW1, 1, kMlpIn, w.h1, B, kMlpHidden, kMlpIn,
                   m->w + kB1, true, st));
    ERQ_TRY(mlp_mm(w.h1, kMlpHidden, 1, m->wb + kW2, 1, kMlpHidden, w.h2, B, kMlpHidden,
                   kMlpHidden, m->w + kB2, true, st));
    ERQ_TRY(mlp_mm(w.h2, kMlpHidden, 1, m->wb + kW3, 1, kMlpHidden, w.z, B, kMlpBins, kMlpHidden,
                   m->w + kB3, false, st));
    return ERQ_OK;
}

// Gradients of the mean cross-entropy into g (parameter layout of mlp.cuh).
erq_status mlp_backward(const erq_probe_model* m, const MlpWork& w, int B, float* g,
                        cudaStream_t st) {
    // output layer
    ERQ_TRY(mlp_mm(w.dz, 1, kMlpBins, w.h2, kMlpHidden, 1, g + kW3, kMlpBins, kMlpHidden, B,
                   (const float*)nullptr, false, st));
    mlp_bias_grad_kernel<<<1, 32, 0, st>>>(w.dz, B, kMlpBins, g + kB3);
    ERQ_TRY(mlp_mm(w.dz, kMlpBins, 1, m->wb + kW3, kMlpHidden, 1, w.dh2, B, kMlpHidden, kMlpBins,
                   (const float*)nullptr, false, st));
    mlp_relu_grad_kernel<<<(unsigned)div_up((uint64_t)B * kMlpHidden, 256), 256, 0, st>>>(
        w.dh2, w.h2, B * kMlpHidden);
    // second layer
    ERQ_TRY(mlp_mm(w.dh2, 1, kMlpHidden, w.h1, kMlpHidden, 1, g + kW2, kMlpHidden, kMlpHidden, B,
                   (const float*)nullptr, false, st));
    mlp_bias_grad_kernel<<<1, kMlpHidden, 0, st>>>(w.dh2, B, kMlpHidden, g + kB2);
    ERQ_TRY(mlp_mm(w.dh2, kMlpHidden, 1, m->wb + kW2, kMlpHidden, 1, w.dh1, B, kMlpHidden,
                   kMlpHidden, (const float*)nullptr, false, st));
    mlp_relu_grad_kernel<<<(unsigned)div_up((uint64_t)B * kMlpHidden, 256), 256, 0, st>>>(
        w.dh1, w.h1, B * kMlpHidden);
    // first layer
    ERQ_TRY(mlp_mm(w.dh1, 1, kMlpHidden, w.x, kMlpIn, 1, g + kW1, kMlpHidden, kMlpIn, B,
                   (const float*)nullptr, false, st));
    mlp_bias_grad_kernel<<<1, kMlpHidden, 0, st>>>(w.dh1, B, kMlpHidden, g + kB1);
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

__global__ void mlp_gather_rows_kernel(const float* __restrict__ X, const uint8_t* __restrict__ y,
                                       const uint32_t* __restrict__ perm, int B,
                                       float* __restrict__ xb, uint8_t* __restrict__ yb) {
    const int r = blockIdx.x;
    if (r >= B) return;
    const uint32_t src = perm[r];
    for (int c = threadIdx.x; c < kMlpIn; c += blockDim.x)
        xb[(size_t)r * kMlpIn + c] = X[(size_t)src * kMlpIn + c];
    if (threadIdx.x == 0) yb[r] = y[src];
}

erq_status model_alloc(erq_probe_model* m) {
    ERQ_CUDA(cudaMalloc(&m->w1d, sizeof(__nv_bfloat16) * kMlpHidden * 2 * kMlpIn));
    ERQ_CUDA(cudaMalloc(&m->w2d, sizeof(__nv_bfloat16) * kMlpHidden * 2 * kMlpHidden));
    ERQ_CUDA(cudaMalloc(&m->w, sizeof(float) * kMlpParams));
    ERQ_CUDA(cudaMalloc(&m->wb, sizeof(__nv_bfloat16) * kMlpParams));
    ERQ_CUDA(cudaMalloc(&m->mean, sizeof(float) * kMlpIn));
    ERQ_CUDA(cudaMalloc(&m->stdv, sizeof(float) * kMlpIn));
    ERQ_CUDA(cudaMalloc(&m->bins_dev, sizeof(int) * kMlpBins));
    return ERQ_OK;
}

erq_status model_dup_weights(erq_probe_model* m, cudaStream_t st) {
    mlp_dup_weights_kernel<<<(unsigned)div_up(kMlpHidden * 2 * kMlpIn, 256), 256, 0, st>>>(
        m->wb, m->w1d, m->w2d);
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}
erq_status model_upload(erq_probe_model* m, const std::vector<float>& w,
                        const std::vector<float>& mean, const std::vector<float>& stdv) {
    ERQ_CUDA(cudaMemcpy(m->w, w.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(m->mean, mean.data(), sizeof(float) * kMlpIn, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(m->stdv, stdv.data(), sizeof(float) * kMlpIn, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(m->bins_dev, m->bins, sizeof(int) * kMlpBins, cudaMemcpyHostToDevice));
    mlp_to_bf16_kernel<<<(unsigned)div_up(kMlpParams, 256), 256>>>(m->w, m->wb, kMlpParams);
    ERQ_CUDA(cudaGetLastError());
    ERQ_TRY(model_dup_weights(m, nullptr));
    ERQ_CUDA(cudaDeviceSynchronize());
    return ERQ_OK;
}

// Forward pass for inference on tensor cores (mlp.cuh): probs[B][8] of raw
// features feats[B][320].  Training and the gradient check use mlp_forward.
erq_status mlp_infer(const erq_probe_model* m, const float* feats, const MlpWork& w, int B,
                     float* probs, cudaStream_t st, bool xs_ready = false) {
    if (B <= 0) return ERQ_OK;
    if (!xs_ready) {
        LaunchTimer t(kMlp, st);
        mlp_standardise_split_kernel<<<(unsigned)div_up((uint64_t)B * kMlpIn, 256), 256, 0, st>>>(
            feats, m->mean, m->stdv, w.xs, B * kMlpIn);
        t.finish();
    }
    {
        GemmEpilogue e;
        e.bias = m->w + kB1;
        e.relu = true;
        ERQ_TRY(gemm_tc(w.xs, m->w1d, w.h1, B, kMlpHidden, 2 * kMlpIn, e, kMlp, st));
    }
    {
        LaunchTimer t(kMlp, st);
        mlp_split_hidden_kernel<<<(unsigned)div_up((uint64_t)B * kMlpHidden, 256), 256, 0, st>>>(
            w.h1, w.hs, B * kMlpHidden);
        t.finish();
    }
    {
        GemmEpilogue e;
        e.bias = m->w + kB2;
        e.relu = true;
        ERQ_TRY(gemm_tc(w.hs, m->w2d, w.h2, B, kMlpHidden, 2 * kMlpHidden, e, kMlp, st));
    }
    {
        LaunchTimer t(kMlp, st);
        mlp_head_kernel<<<(unsigned)div_up(B, 256 / kMlpBins), 256, 0, st>>>(w.h2, m->wb + kW3,
                                                                           m->w + kB3, B, probs);
        t.finish();
    }
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

// Probe features of a batch of rotated queries on the device.
// With a model and xs, also its standardised first-layer input.
erq_status features_device(const erq_index* idx, const Batch& b, uint64_t nprobe, float* near_d,
                           float* feats, cudaStream_t st, const erq_probe_model* m = nullptr,
                           __nv_bfloat16* xs = nullptr, bool* split = nullptr) {
    ERQ_TRY(launch_probe_tc(idx, b, nprobe, st, near_d, split));
    LaunchTimer t(kMlp, st);
    probe_features_kernel<<<(unsigned)b.nq, 128, 0, st>>>(
        b.qrot, (int)idx->D, b.qn, near_d, (int)b.nq, feats, m && xs ? m->mean : nullptr,
        m && xs ? m->stdv : nullptr, m ? xs : nullptr);
    t.finish();
    ERQ_CUDA(cudaGetLastError());
    return ERQ_OK;
}

}  // namespace

// ------------------------------------------------------------- k-means
// splitmix64 (Steele, Lea and Flood, 2014): the random stream of the
// k-means initialisation and of its empty-cluster splits.
uint64_t splitmix64_next(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double splitmix64_uniform(uint64_t& s) {  // in [0, 1), 53 random bits
    return (double)(splitmix64_next(s) >> 11) * (1.0 / 9007199254740992.0);
}

// A D x D orthogonal matrix for erq_build_index when the caller gives none:
// Householder QR (double) of a matrix of standard normal samples (Box-Muller
// on the splitmix64 stream), P = Q^T with the signs that make R's diagonal
// positive.  Any orthogonal rotation serves the quantiser (the reference
// draws its own, inc/index/Rotator.hpp:14-19).
void random_rotation(uint64_t D, uint64_t seed, std::vector<float>& P) {
    uint64_t s = seed;
    std::vector<double> a(D * D);
    for (uint64_t i = 0; i < D * D; i += 2) {
        const double u1 = 1.0 - splitmix64_uniform(s), u2 = splitmix64_uniform(s);
        const double r = std::sqrt(-2.0 * std::log(u1));
        a[i] = r * std::cos(6.283185307179586 * u2);
        if (i + 1 < D * D) a[i + 1] = r * std::sin(6.283185307179586 * u2);
    }
    // reflector k: v = column k of a from row k down (after the update), tau
    std::vector<double> tau(D, 0.0), rdiag(D, 0.0), dot(D);
    auto reflect = [&](std::vector<double>& m, uint64_t kk, uint64_t j0) {
        std::fill(dot.begin() + j0, dot.end(), 0.0);
        for (uint64_t i = kk; i < D; ++i) {
            const double vi = a[i * D + kk];
            for (uint64_t j = j0; j < D; ++j) dot[j] += vi * m[i * D + j];
        }
        for (uint64_t i = kk; i < D; ++i) {
            const double vi = a[i * D + kk] * tau[kk];
            for (uint64_t j = j0; j < D; ++j) m[i * D + j] -= dot[j] * vi;
        }
    };
    for (uint64_t kk = 0; kk < D; ++kk) {
        double norm = 0;
        for (uint64_t i = kk; i < D; ++i) norm += a[i * D + kk] * a[i * D + kk];
        norm = std::sqrt(norm);
        const double alpha = a[kk * D + kk] > 0 ? -norm : norm;
        rdiag[kk] = alpha;
        a[kk * D + kk] -= alpha;
        double v2 = 0;
        for (uint64_t i = kk; i < D; ++i) v2 += a[i * D + kk] * a[i * D + kk];
        tau[kk] = v2 > 0 ? 2.0 / v2 : 0.0;
        if (kk + 1 < D) reflect(a, kk, kk + 1);
    }
    std::vector<double> q(D * D, 0.0);  // Q = H_0 H_1 ... H_{D-1}
    for (uint64_t i = 0; i < D; ++i) q[i * D + i] = 1.0;
    for (uint64_t kk = D; kk-- > 0;) reflect(q, kk, 0);
    // P = Q^T with column signs making R's diagonal positive
    P.resize(D * D);
    for (uint64_t i = 0; i < D; ++i)
        for (uint64_t j = 0; j < D; ++j) P[j * D + i] = (float)(rdiag[j] < 0 ? -q[i * D + j] : q[i * D + j]);
}

// Device buffers of one clustering run, freed on scope exit.
struct KmBuffers {
    std::vector<void*> owned;
    template <typename T>
    erq_status alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16));
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? ERQ_ERR_OUT_OF_MEMORY : ERQ_ERR_CUDA,
                        "cudaMalloc(%zu bytes) for k-means failed: %s", count * sizeof(T),
                        cudaGetErrorString(e));
        owned.push_back(q);
        *p = static_cast<T*>(q);
        return ERQ_OK;
    }
    ~KmBuffers() {
        for (void* q : owned) cudaFree(q);
    }
};

// Lloyd iterations (kmeans.cuh).  cent: device [k][dim], updated in place;
// rng: the split stream; counts_host: the last iteration's cluster sizes
// before its splits (optional); final_assign: one more assignment to the
// final centroids.
erq_status km_iterate(const float* x, uint64_t n, uint64_t dim, uint64_t k, int iters, float* cent,
                      uint32_t* assign, uint64_t& rng, uint32_t* counts_host, bool final_assign,
                      cudaStream_t st) {
    const uint64_t Cp = (dim + 63) / 64 * 64;
    const uint64_t R = std::min<uint64_t>(n, std::max<uint64_t>(1024, (256ull << 20) / std::max<uint64_t>(k, 1)));
    KmBuffers b;
    __nv_bfloat16 *c_split = nullptr, *x_split = nullptr;
    float *cn = nullptr, *xn = nullptr, *dist = nullptr;
    unsigned long long* sums = nullptr;
    uint32_t* counts = nullptr;
    unsigned* amax = nullptr;
    ERQ_TRY(b.alloc(&c_split, k * 3 * Cp));
    ERQ_TRY(b.alloc(&cn, k));
    ERQ_TRY(b.alloc(&x_split, R * 3 * Cp));
    ERQ_TRY(b.alloc(&xn, R));
    ERQ_TRY(b.alloc(&dist, R * k));
    ERQ_TRY(b.alloc(&sums, k * dim));
    ERQ_TRY(b.alloc(&counts, k));
    ERQ_TRY(b.alloc(&amax, 1));
    // fixed-point scale 2^s: n * max|x| * 2^s < 2^62, s <= 32
    ERQ_CUDA(cudaMemsetAsync(amax, 0, sizeof(unsigned), st));
    abs_max_kernel<<<1184, 256, 0, st>>>(x, n * dim, amax);
    ERQ_CUDA(cudaGetLastError());
    unsigned amax_bits = 0;
    ERQ_CUDA(cudaMemcpyAsync(&amax_bits, amax, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaStreamSynchronize(st));
    float amax_f = 0.f;
    std::memcpy(&amax_f, &amax_bits, sizeof(float));
    const double top = std::max(1e-30, (double)amax_f) * (double)n;
    const double scale = std::ldexp(1.0, std::min(32, (int)std::floor(61.0 - std::log2(top))));
    std::vector<uint32_t> cnt(k);
    auto assign_all = [&]() -> erq_status {
        split_rows_kernel<<<(unsigned)k, 256, 0, st>>>(cent, (int)k, (int)dim, (int)Cp, false, c_split, cn);
        ERQ_CUDA(cudaGetLastError());
        for (uint64_t r0 = 0; r0 < n; r0 += R) {
            const uint64_t rows = std::min(R, n - r0);
            split_rows_kernel<<<(unsigned)rows, 256, 0, st>>>(x + r0 * dim, (int)rows, (int)dim, (int)Cp,
                                                              true, x_split, xn);
            ERQ_CUDA(cudaGetLastError());
            GemmEpilogue epi;
            epi.row_norm = xn;
            epi.col_norm = cn;
            ERQ_TRY(gemm_tc(x_split, c_split, dist, (int)rows, (int)k, (int)(3 * Cp), epi, kGemm, st));
            argmin_rows_kernel<<<(unsigned)div_up(rows * 32, 256), 256, 0, st>>>(dist, (int)rows, (int)k,
                                                                                 assign + r0);
            ERQ_CUDA(cudaGetLastError());
        }
        return ERQ_OK;
    };
    for (int it = 0; it < iters; ++it) {
        ERQ_TRY(assign_all());
        ERQ_CUDA(cudaMemsetAsync(sums, 0, k * dim * sizeof(unsigned long long), st));
        ERQ_CUDA(cudaMemsetAsync(counts, 0, k * sizeof(uint32_t), st));
        kmeans_accumulate_kernel<<<(unsigned)div_up(n, 8), 256, 0, st>>>(x, (int)n, (int)dim, scale,
                                                                          assign, sums, counts);
        ERQ_CUDA(cudaGetLastError());
        kmeans_update_kernel<<<1184, 256, 0, st>>>(sums, counts, (int)k, (int)dim, scale, cent);
        ERQ_CUDA(cudaGetLastError());
        ERQ_CUDA(cudaMemcpyAsync(cnt.data(), counts, k * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        ERQ_CUDA(cudaStreamSynchronize(st));
        ERQ_TRY(tc_status_check_now());
        if (counts_host) std::copy(cnt.begin(), cnt.end(), counts_host);
        // empty clusters: split a populated one, chosen with probability
        // proportional to (size - 1)
        std::vector<double> c(cnt.begin(), cnt.end());
        for (uint64_t ci = 0; ci < k; ++ci) {
            if (c[ci] != 0) continue;
            double total = 0;
            for (uint64_t j = 0; j < k; ++j) total += std::max(c[j] - 1.0, 0.0);
            uint64_t cj = 0;
            if (total > 0) {
                const double u = splitmix64_uniform(rng) * total;
                double run = 0;
                for (cj = 0; cj + 1 < k; ++cj) {
                    run += std::max(c[cj] - 1.0, 0.0);
                    if (u < run) break;
                }
            } else {
                cj = (uint64_t)(std::max_element(c.begin(), c.end()) - c.begin());
            }
            kmeans_split_kernel<<<(unsigned)div_up(dim, 256), 256, 0, st>>>(cent, (int)dim, (int)ci,
                                                                            (int)cj, 1.f / 1024.f);
            ERQ_CUDA(cudaGetLastError());
            c[ci] = std::floor(c[cj] / 2);
            c[cj] -= c[ci];
        }
    }
    if (final_assign) ERQ_TRY(assign_all());
    ERQ_CUDA(cudaStreamSynchronize(st));
    ERQ_TRY(tc_status_check_now());
    return ERQ_OK;
}

// ------------------------------------------------- allocation-free search
// Scratch of erq_search_noalloc: one fixed array in this module's device
// memory (every GPU that loads the library holds it until the process
// exits).  Host code must not take its address with &; the device address is
// fetched once per device with cudaGetSymbolAddress.
constexpr uint64_t kNoAllocScratchBytes = 64ull << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mu;
uint8_t* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device`, which must be current.
erq_status noalloc_scratch(int device, uint8_t** out) {
    if (device < 0 || device >= kMaxDevices)
        return fail(ERQ_ERR_UNSUPPORTED, "device ordinal %d above %d", device, kMaxDevices - 1);
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        ERQ_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[device] = static_cast<uint8_t*>(p);
    }
    *out = g_noalloc_ptr[device];
    return ERQ_OK;
}

uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

// Scratch bytes one call needs for nq queries at this nprobe.
// Sort keys per query of the exact probe beyond shared memory (0: none).
uint64_t noalloc_sort_cap(const erq_index* idx, uint64_t nprobe) {
    const int npow2 = next_pow2((int)std::min<uint64_t>(nprobe, idx->K));
    return npow2 > kProbeSortSmemKeys ? (uint64_t)npow2 : 0;
}

uint64_t noalloc_bytes(const erq_index* idx, uint64_t nq, uint64_t nprobe) {
    const uint64_t np = nq * nprobe;
    return align256(nq * idx->K * 4) + 2 * align256(np * 4) + align256(np * 8) +
           align256(nq * 32ull * idx->top_blocks[nprobe] * 4) + 3 * align256(np * 4) +
           align256(nq * noalloc_sort_cap(idx, nprobe) * 8);
}
}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

int erq_version(void) { return ERQ_API_VERSION; }

const char* erq_status_string(erq_status s) {
    switch (s) {
        case ERQ_OK: return "ok";
        case ERQ_ERR_INVALID_ARGUMENT: return "invalid argument";
        case ERQ_ERR_IO: return "i/o error";
        case ERQ_ERR_FORMAT: return "bad index format";
        case ERQ_ERR_UNSUPPORTED: return "unsupported";
        case ERQ_ERR_CUDA: return "cuda error";
        case ERQ_ERR_OUT_OF_MEMORY: return "out of memory";
        case ERQ_ERR_TIMEOUT: return "timeout";
    }
    return "unknown status";
}

const char* erq_last_error(void) { return g_last_error.c_str(); }

erq_status erq_index_load(const char* path, int device, erq_index** out) {
    if (!out) return fail(ERQ_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!path) return fail(ERQ_ERR_INVALID_ARGUMENT, "path is NULL");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(ERQ_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= ndev)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "device %d outside [0, %d)", device, ndev);
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    std::unique_ptr<erq_index> idx(new (std::nothrow) erq_index());
    if (!idx) return fail(ERQ_ERR_OUT_OF_MEMORY, "host allocation failed");
    idx->device = device;
    ERQ_TRY(load_impl(path, idx.get()));
    *out = idx.release();
    return ERQ_OK;
}

erq_status erq_index_get_info(const erq_index* idx, erq_index_info* info) {
    if (!idx || !info) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    info->n = idx->N;
    info->dim = idx->DIM;
    info->padded_dim = idx->D;
    info->num_clusters = idx->K;
    info->ex_bits = idx->EX;
    info->device_bytes = idx->device_bytes;
    info->device = idx->device;
    info->block_factors = idx->factors;
    return ERQ_OK;
}

void erq_index_free(erq_index* idx) { delete idx; }

erq_status erq_rotate(const erq_index* idx, const float* queries, uint64_t nq, float* rotated,
                      void* stream) {
    if (!idx) return fail(ERQ_ERR_INVALID_ARGUMENT, "index is NULL");
    if (nq == 0) return ERQ_OK;
    if (!queries || !rotated) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL buffer");
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool q_dev = is_device_ptr(queries), o_dev = is_device_ptr(rotated);
    Scratch s(st, idx->pool);
    const float* qin = queries;
    float* out = rotated;
    if (!q_dev) {
        float* tmp = nullptr;
        ERQ_TRY(s.alloc(&tmp, nq * idx->DIM));
        ERQ_CUDA(cudaMemcpyAsync(tmp, queries, nq * idx->DIM * 4, cudaMemcpyHostToDevice, st));
        qin = tmp;
    }
    if (!o_dev) ERQ_TRY(s.alloc(&out, nq * idx->D));
    ERQ_TRY(rotate_device(idx, qin, nq, out, st));
    if (!o_dev) {
        ERQ_CUDA(cudaMemcpyAsync(rotated, out, nq * idx->D * 4, cudaMemcpyDeviceToHost, st));
        ERQ_CUDA(cudaStreamSynchronize(st));
    } else if (!q_dev) {
        ERQ_CUDA(cudaStreamSynchronize(st));
    }
    return ERQ_OK;
}

erq_status erq_search(const erq_index* idx, const float* rotated_queries, uint64_t nq, uint64_t k,
                      uint64_t nprobe, uint32_t* ids, float* dists, void* stream) {
    return search_entry(idx, rotated_queries, true, nq, k, nprobe, ids, dists, stream);
}

erq_status erq_search_raw(const erq_index* idx, const float* queries, uint64_t nq, uint64_t k,
                          uint64_t nprobe, uint32_t* ids, float* dists, void* stream) {
    return search_entry(idx, queries, false, nq, k, nprobe, ids, dists, stream);
}

erq_status erq_search_noalloc(const erq_index* idx, const float* rotated_queries, uint64_t nq,
                              uint64_t k, uint64_t nprobe, uint32_t* ids, float* dists,
                              void* stream) {
    ERQ_TRY(check_search_args(idx, nq, k, nprobe, rotated_queries, ids));
    if (nq == 0) return ERQ_OK;
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    if (!is_device_ptr(rotated_queries) || !is_device_ptr(ids) || (dists && !is_device_ptr(dists)))
        return fail(ERQ_ERR_INVALID_ARGUMENT,
                    "erq_search_noalloc takes device memory only (queries, ids, dists)");
    if ((reinterpret_cast<uintptr_t>(rotated_queries) & 15) ||
        (reinterpret_cast<uintptr_t>(ids) & 3) || (reinterpret_cast<uintptr_t>(dists) & 3))
        return fail(ERQ_ERR_INVALID_ARGUMENT,
                    "queries must be 16-byte aligned and ids/dists 4-byte aligned");
    const uint64_t need = noalloc_bytes(idx, nq, nprobe);
    if (need > kNoAllocScratchBytes) {
        // largest batch that fits: noalloc_bytes grows with nq, so bisect
        uint64_t fit = 0, hi = nq;  // noalloc_bytes(fit) fits, noalloc_bytes(hi) does not
        while (hi - fit > 1) {
            const uint64_t mid = fit + (hi - fit) / 2;
            if (noalloc_bytes(idx, mid, nprobe) <= kNoAllocScratchBytes) fit = mid; else hi = mid;
        }
        return fail(ERQ_ERR_INVALID_ARGUMENT,
                    "%llu queries at nprobe=%llu need %llu bytes of scratch; the static scratch "
                    "holds %llu bytes (at most %llu queries per call here)",
                    (unsigned long long)nq, (unsigned long long)nprobe, (unsigned long long)need,
                    (unsigned long long)kNoAllocScratchBytes, (unsigned long long)fit);
    }
    uint8_t* base = nullptr;
    ERQ_TRY(noalloc_scratch(idx->device, &base));
    ERQ_TRY(configure_kernels((int)idx->D, (int)idx->K, (int)k));
    // Carve the batch buffers.  Every element a kernel reads is written
    // earlier in the same call, so nothing needs clearing between calls.
    const uint64_t np = nq * nprobe;
    Batch b;
    b.nq = nq;
    b.qrot = rotated_queries;
    uint8_t* cur = base;
    auto take = [&cur](uint64_t bytes) {
        uint8_t* p = cur;
        cur += align256(bytes);
        return p;
    };
    b.dist = reinterpret_cast<float*>(take(nq * idx->K * 4));
    b.probe_cid = reinterpret_cast<uint32_t*>(take(np * 4));
    b.probe_sqy = reinterpret_cast<float*>(take(np * 4));
    b.s_off = reinterpret_cast<uint64_t*>(take(np * 8));
    b.S = reinterpret_cast<int32_t*>(take(nq * 32ull * idx->top_blocks[nprobe] * 4));
    b.delta = reinterpret_cast<float*>(take(np * 4));
    b.sumq = reinterpret_cast<float*>(take(np * 4));
    b.vl = reinterpret_cast<float*>(take(np * 4));
    b.sort_cap = noalloc_sort_cap(idx, nprobe);
    if (b.sort_cap) b.sortbuf = reinterpret_cast<uint64_t*>(take(nq * b.sort_cap * 8));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ERQ_TRY(launch_probe(idx, b, nprobe, st));
    ERQ_TRY(launch_scan(idx, b, nprobe, st));
    ERQ_TRY(launch_refine(idx, b, nprobe, k, ids, dists, st));
    return ERQ_OK;
}

// ------------------------------------------------------------- debug ABI
erq_status erq_debug_probe(const erq_index* idx, const float* qrot, uint64_t nq, uint64_t nprobe,
                           uint32_t* cids, float* sqr_y) {
    if (!idx || !qrot || !cids || !sqr_y) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (nprobe < 1 || nprobe > idx->K) return fail(ERQ_ERR_INVALID_ARGUMENT, "bad nprobe");
    if (nq == 0) return ERQ_OK;
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    ERQ_TRY(configure_kernels((int)idx->D, (int)idx->K, 1));
    cudaStream_t st = 0;
    Scratch s(st, idx->pool);
    float* q = nullptr;
    ERQ_TRY(s.alloc(&q, nq * idx->D));
    ERQ_CUDA(cudaMemcpyAsync(q, qrot, nq * idx->D * 4, cudaMemcpyHostToDevice, st));
    Batch b;
    ERQ_TRY(alloc_batch(s, idx, nq, nprobe, b));
    b.qrot = q;
    ERQ_TRY(launch_probe_tc(idx, b, nprobe, st));
    ERQ_CUDA(cudaMemcpyAsync(cids, b.probe_cid, nq * nprobe * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaMemcpyAsync(sqr_y, b.probe_sqy, nq * nprobe * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaStreamSynchronize(st));
    return ERQ_OK;
}

erq_status erq_debug_centroid_dists(const erq_index* idx, const float* qrot, uint64_t nq,
                                    float* dist) {
    if (!idx || !qrot || !dist) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (nq == 0) return ERQ_OK;
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    cudaStream_t st = 0;
    Scratch s(st, idx->pool);
    float* q = nullptr;
    float* d = nullptr;
    if (div_up(nq, kCdTQ) > 65535)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "at most %llu queries per call",
                    (unsigned long long)(65535ull * kCdTQ));
    ERQ_TRY(s.alloc(&q, nq * idx->D));
    ERQ_TRY(s.alloc(&d, nq * idx->K));
    ERQ_CUDA(cudaMemcpyAsync(q, qrot, nq * idx->D * 4, cudaMemcpyHostToDevice, st));
    dim3 g1((unsigned)div_up(idx->K, kCdTC), (unsigned)div_up(nq, kCdTQ));
    centroid_dist_kernel<<<g1, 256, 0, st>>>(q, (int)nq, idx->centroids, (int)idx->K, (int)idx->D, d);
    ERQ_CUDA(cudaGetLastError());
    ERQ_CUDA(cudaMemcpyAsync(dist, d, nq * idx->K * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaStreamSynchronize(st));
    return ERQ_OK;
}

uint64_t erq_debug_scan_capacity(const erq_index* idx, uint64_t nq, uint64_t nprobe) {
    if (!idx || nprobe > idx->K) return 0;
    return nq * 32ull * idx->top_blocks[nprobe];
}

erq_status erq_debug_scan(const erq_index* idx, const float* qrot, uint64_t nq, uint64_t nprobe,
                          uint32_t* cids, float* sqr_y, float* delta, float* sumq,
                          uint64_t* s_offsets, int32_t* S, uint64_t s_capacity) {
    if (!idx || !qrot || !cids || !sqr_y || !delta || !sumq || !s_offsets || !S)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (nprobe < 1 || nprobe > idx->K) return fail(ERQ_ERR_INVALID_ARGUMENT, "bad nprobe");
    if (nq == 0) return ERQ_OK;
    const uint64_t need = nq * 32ull * idx->top_blocks[nprobe];
    if (s_capacity < need)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "S capacity %llu < %llu",
                    (unsigned long long)s_capacity, (unsigned long long)need);
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    ERQ_TRY(configure_kernels((int)idx->D, (int)idx->K, 1));
    cudaStream_t st = 0;
    Scratch s(st, idx->pool);
    float* q = nullptr;
    ERQ_TRY(s.alloc(&q, nq * idx->D));
    ERQ_CUDA(cudaMemcpyAsync(q, qrot, nq * idx->D * 4, cudaMemcpyHostToDevice, st));
    Batch b;
    ERQ_TRY(alloc_batch(s, idx, nq, nprobe, b));
    b.qrot = q;
    ERQ_CUDA(cudaMemsetAsync(b.S, 0, need * 4, st));
    ERQ_TRY(launch_probe_tc(idx, b, nprobe, st));
    ERQ_TRY(launch_scan(idx, b, nprobe, st));
    const uint64_t np = nq * nprobe;
    ERQ_CUDA(cudaMemcpyAsync(cids, b.probe_cid, np * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaMemcpyAsync(sqr_y, b.probe_sqy, np * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaMemcpyAsync(delta, b.delta, np * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaMemcpyAsync(sumq, b.sumq, np * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaMemcpyAsync(s_offsets, b.s_off, np * 8, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaMemcpyAsync(S, b.S, need * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaStreamSynchronize(st));
    return ERQ_OK;
}


// ------------------------------------------------------------ learned probing
erq_status erq_probe_features(const erq_index* idx, const float* rotated_queries, uint64_t nq,
                              float* features, void* stream) {
    if (!idx || !rotated_queries || !features) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (nq == 0) return ERQ_OK;
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    ERQ_TRY(configure_kernels((int)idx->D, (int)idx->K, 1));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool q_dev = is_device_ptr(rotated_queries), f_dev = is_device_ptr(features);
    Scratch s(st, idx->pool);
    const float* q = rotated_queries;
    if (!q_dev || (reinterpret_cast<uintptr_t>(q) & 15)) {
        float* tmp = nullptr;
        ERQ_TRY(s.alloc(&tmp, nq * idx->D));
        ERQ_CUDA(cudaMemcpyAsync(tmp, rotated_queries, nq * idx->D * 4, cudaMemcpyDefault, st));
        q = tmp;
    }
    float* fout = features;
    if (!f_dev) ERQ_TRY(s.alloc(&fout, nq * kMlpIn));
    const uint64_t nprobe = 1;
    const uint64_t bq = batch_queries(idx, std::max<uint64_t>(nprobe, 1), nq);
    Batch b;
    ERQ_TRY(alloc_batch(s, idx, bq, nprobe, b));
    ERQ_TRY(alloc_probe_lists(s, bq, b));
    float* near_d = nullptr;
    ERQ_TRY(s.alloc(&near_d, bq * kFeatDists));
    for (uint64_t q0 = 0; q0 < nq; q0 += bq) {
        b.nq = std::min(bq, nq - q0);
        b.qrot = q + q0 * idx->D;
        bool split = false;  // the features need no probe list: a split probe stops there
        ERQ_TRY(features_device(idx, b, nprobe, near_d, fout + q0 * kMlpIn, st, nullptr, nullptr, &split));
    }
    if (!f_dev) {
        ERQ_CUDA(cudaMemcpyAsync(features, fout, nq * kMlpIn * 4, cudaMemcpyDeviceToHost, st));
        ERQ_CUDA(cudaStreamSynchronize(st));
    } else if (!q_dev) {
        ERQ_CUDA(cudaStreamSynchronize(st));
    }
    return ERQ_OK;
}

erq_status erq_probe_model_train(const float* features, const uint8_t* labels, uint64_t n,
                                 const uint32_t* bin_nprobe, int epochs, int batch, float lr,
                                 uint64_t seed, int device, erq_probe_model** out,
                                 float* final_loss) {
    if (!features || !labels || !bin_nprobe || !out) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (n < 2 || epochs < 1 || batch < 1 || !(lr > 0.f))
        return fail(ERQ_ERR_INVALID_ARGUMENT, "need n >= 2, epochs >= 1, batch >= 1, lr > 0");
    for (int j = 0; j < kMlpBins; ++j)
        if (bin_nprobe[j] < 1 || (j > 0 && bin_nprobe[j] <= bin_nprobe[j - 1]))
            return fail(ERQ_ERR_INVALID_ARGUMENT, "bin_nprobe must be increasing and >= 1");
    for (uint64_t i = 0; i < n; ++i)
        if (labels[i] >= kMlpBins) return fail(ERQ_ERR_INVALID_ARGUMENT, "label >= %d", kMlpBins);
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    std::unique_ptr<erq_probe_model> m(new (std::nothrow) erq_probe_model());
    if (!m) return fail(ERQ_ERR_OUT_OF_MEMORY, "host allocation failed");
    m->device = device;
    for (int j = 0; j < kMlpBins; ++j) m->bins[j] = (int)bin_nprobe[j];
    ERQ_TRY(model_alloc(m.get()));
    // standardisation statistics (float64 on the host)
    std::vector<double> mu(kMlpIn, 0.0), var(kMlpIn, 0.0);
    for (uint64_t i = 0; i < n; ++i)
        for (int c = 0; c < kMlpIn; ++c) mu[c] += features[i * kMlpIn + c];
    for (int c = 0; c < kMlpIn; ++c) mu[c] /= (double)n;
    for (uint64_t i = 0; i < n; ++i)
        for (int c = 0; c < kMlpIn; ++c) {
            const double d = features[i * kMlpIn + c] - mu[c];
            var[c] += d * d;
        }
    std::vector<float> mean(kMlpIn), stdv(kMlpIn);
    for (int c = 0; c < kMlpIn; ++c) {
        mean[c] = (float)mu[c];
        stdv[c] = (float)std::max(std::sqrt(var[c] / (double)n), 1e-6);
    }
    // initial weights: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)), zero biases
    std::mt19937_64 rng(seed);
    std::vector<float> w(kMlpParams, 0.f);
    auto init = [&](int off, int rows, int cols) {
        std::uniform_real_distribution<float> u(-1.f / std::sqrt((float)cols), 1.f / std::sqrt((float)cols));
        for (int i = 0; i < rows * cols; ++i) w[off + i] = u(rng);
    };
    init(kW1, kMlpHidden, kMlpIn);
    init(kW2, kMlpHidden, kMlpHidden);
    init(kW3, kMlpBins, kMlpHidden);
    ERQ_TRY(model_upload(m.get(), w, mean, stdv));
    // the whole standardised training set on the device
    cudaStream_t st = nullptr;
    ERQ_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamCloser {
        cudaStream_t s;
        ~StreamCloser() { cudaStreamDestroy(s); }
    } closer{st};
    float *X = nullptr, *Xraw = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    uint8_t *Y = nullptr, *yb = nullptr;
    uint32_t* perm_d = nullptr;
    struct Frees {
        std::vector<void*> p;
        ~Frees() {
            for (void* x : p) cudaFree(x);
        }
    } frees;
    auto dmalloc = [&](void** p, size_t bytes) -> erq_status {
        ERQ_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 16)));
        frees.p.push_back(*p);
        return ERQ_OK;
    };
    ERQ_TRY(dmalloc((void**)&Xraw, n * kMlpIn * 4));
    ERQ_TRY(dmalloc((void**)&X, n * kMlpIn * 4));
    ERQ_TRY(dmalloc((void**)&Y, n));
    ERQ_TRY(dmalloc((void**)&g, kMlpParams * 4));
    ERQ_TRY(dmalloc((void**)&m1, kMlpParams * 4));
    ERQ_TRY(dmalloc((void**)&m2, kMlpParams * 4));
    ERQ_TRY(dmalloc((void**)&perm_d, n * 4));
    ERQ_TRY(dmalloc((void**)&yb, (size_t)batch));
    ERQ_CUDA(cudaMemcpy(Xraw, features, n * kMlpIn * 4, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(Y, labels, n, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemsetAsync(m1, 0, kMlpParams * 4, st));
    ERQ_CUDA(cudaMemsetAsync(m2, 0, kMlpParams * 4, st));
    mlp_standardise_kernel<<<(unsigned)div_up(n * kMlpIn, 256), 256, 0, st>>>(Xraw, m->mean, m->stdv,
                                                                            X, (int)(n * kMlpIn));
    ERQ_CUDA(cudaGetLastError());
    MlpWork wk;
    {
        float* p = nullptr;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpIn * 4)); wk.x = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpHidden * 4)); wk.h1 = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpHidden * 4)); wk.h2 = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpBins * 4)); wk.z = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpBins * 4)); wk.probs = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpBins * 4)); wk.dz = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpHidden * 4)); wk.dh2 = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * kMlpHidden * 4)); wk.dh1 = p;
        ERQ_TRY(dmalloc((void**)&p, (size_t)batch * 4)); wk.loss = p;
    }
    std::vector<uint32_t> perm(n);
    std::vector<float> loss_h(batch);
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    int t = 0;
    double last = 0.0;
    for (int e = 0; e < epochs; ++e) {
        std::iota(perm.begin(), perm.end(), 0u);
        std::shuffle(perm.begin(), perm.end(), rng);
        ERQ_CUDA(cudaMemcpyAsync(perm_d, perm.data(), n * 4, cudaMemcpyHostToDevice, st));
        double sum = 0.0;
        uint64_t seen = 0;
        for (uint64_t b0 = 0; b0 + 1 < n; b0 += batch) {
            const int B = (int)std::min<uint64_t>(batch, n - b0);
            mlp_gather_rows_kernel<<<B, 128, 0, st>>>(X, Y, perm_d + b0, B, wk.x, yb);
            ERQ_TRY(mlp_forward(m.get(), wk, B, st));
            mlp_softmax_xent_kernel<<<(unsigned)div_up(B, 128), 128, 0, st>>>(wk.z, yb, B, wk.probs,
                                                                             wk.dz, wk.loss);
            ERQ_TRY(mlp_backward(m.get(), wk, B, g, st));
            ++t;
            const float bc1 = 1.f - std::pow(beta1, (float)t), bc2 = 1.f - std::pow(beta2, (float)t);
            mlp_adam_kernel<<<(unsigned)div_up(kMlpParams, 256), 256, 0, st>>>(
                m->w, g, m1, m2, m->wb, kMlpParams, lr, beta1, beta2, eps, bc1, bc2);
            ERQ_CUDA(cudaGetLastError());
            if (e == epochs - 1) {
                ERQ_CUDA(cudaMemcpyAsync(loss_h.data(), wk.loss, B * 4, cudaMemcpyDeviceToHost, st));
                ERQ_CUDA(cudaStreamSynchronize(st));
                for (int r = 0; r < B; ++r) sum += loss_h[r];
                seen += B;
            }
        }
        if (e == epochs - 1) last = seen ? sum / seen : 0.0;
    }
    ERQ_TRY(model_dup_weights(m.get(), st));
    ERQ_CUDA(cudaStreamSynchronize(st));
    if (final_loss) *final_loss = (float)last;
    *out = m.release();
    return ERQ_OK;
}

static const char kModelMagic[8] = {'E', 'R', 'Q', 'P', 'R', 'O', 'B', '1'};

erq_status erq_probe_model_save(const erq_probe_model* m, const char* path) {
    if (!m || !path) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard guard;
    ERQ_TRY(guard.set(m->device));
    std::vector<float> w(kMlpParams), mean(kMlpIn), stdv(kMlpIn);
    ERQ_CUDA(cudaMemcpy(w.data(), m->w, kMlpParams * 4, cudaMemcpyDeviceToHost));
    ERQ_CUDA(cudaMemcpy(mean.data(), m->mean, kMlpIn * 4, cudaMemcpyDeviceToHost));
    ERQ_CUDA(cudaMemcpy(stdv.data(), m->stdv, kMlpIn * 4, cudaMemcpyDeviceToHost));
    std::unique_ptr<FILE, FileCloser> f(fopen(path, "wb"));
    if (!f) return fail(ERQ_ERR_IO, "cannot write '%s'", path);
    const int32_t dims[3] = {kMlpIn, kMlpHidden, kMlpBins};
    bool ok = fwrite(kModelMagic, 1, 8, f.get()) == 8 && fwrite(dims, 4, 3, f.get()) == 3 &&
              fwrite(m->bins, 4, kMlpBins, f.get()) == (size_t)kMlpBins &&
              fwrite(mean.data(), 4, kMlpIn, f.get()) == (size_t)kMlpIn &&
              fwrite(stdv.data(), 4, kMlpIn, f.get()) == (size_t)kMlpIn &&
              fwrite(w.data(), 4, kMlpParams, f.get()) == (size_t)kMlpParams;
    return ok ? ERQ_OK : fail(ERQ_ERR_IO, "short write to '%s'", path);
}

erq_status erq_probe_model_load(const char* path, int device, erq_probe_model** out) {
    if (!path || !out) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    std::unique_ptr<FILE, FileCloser> f(fopen(path, "rb"));
    if (!f) return fail(ERQ_ERR_IO, "cannot open '%s'", path);
    char magic[8];
    int32_t dims[3];
    std::unique_ptr<erq_probe_model> m(new (std::nothrow) erq_probe_model());
    if (!m) return fail(ERQ_ERR_OUT_OF_MEMORY, "host allocation failed");
    std::vector<float> w(kMlpParams), mean(kMlpIn), stdv(kMlpIn);
    if (fread(magic, 1, 8, f.get()) != 8 || memcmp(magic, kModelMagic, 8) != 0)
        return fail(ERQ_ERR_FORMAT, "'%s' is not a probe model", path);
    if (fread(dims, 4, 3, f.get()) != 3 || dims[0] != kMlpIn || dims[1] != kMlpHidden ||
        dims[2] != kMlpBins)
        return fail(ERQ_ERR_FORMAT, "probe model dimensions do not match");
    if (fread(m->bins, 4, kMlpBins, f.get()) != (size_t)kMlpBins ||
        fread(mean.data(), 4, kMlpIn, f.get()) != (size_t)kMlpIn ||
        fread(stdv.data(), 4, kMlpIn, f.get()) != (size_t)kMlpIn ||
        fread(w.data(), 4, kMlpParams, f.get()) != (size_t)kMlpParams)
        return fail(ERQ_ERR_FORMAT, "probe model file truncated");
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    m->device = device;
    ERQ_TRY(model_alloc(m.get()));
    ERQ_TRY(model_upload(m.get(), w, mean, stdv));
    *out = m.release();
    return ERQ_OK;
}

void erq_probe_model_free(erq_probe_model* m) { delete m; }

erq_status erq_probe_model_predict(const erq_probe_model* m, const float* features, uint64_t n,
                                   float* probs, void* stream) {
    if (!m || !features || !probs) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0) return ERQ_OK;
    DeviceGuard guard;
    ERQ_TRY(guard.set(m->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float *fin = nullptr, *pout = nullptr;
    std::vector<void*> owned;
    struct Frees {
        std::vector<void*>& p;
        ~Frees() {
            for (void* x : p) cudaFree(x);
        }
    } frees{owned};
    const bool f_dev = is_device_ptr(features), p_dev = is_device_ptr(probs);
    if (!f_dev) {
        ERQ_CUDA(cudaMalloc(&fin, n * kMlpIn * 4));
        owned.push_back(fin);
        ERQ_CUDA(cudaMemcpyAsync(fin, features, n * kMlpIn * 4, cudaMemcpyHostToDevice, st));
    } else {
        fin = const_cast<float*>(features);
    }
    if (!p_dev) {
        ERQ_CUDA(cudaMalloc(&pout, n * kMlpBins * 4));
        owned.push_back(pout);
    } else {
        pout = probs;
    }
    MlpWork wk;
    for (float** p : {&wk.h1, &wk.h2, &wk.z}) {
        const size_t cols = p == &wk.z ? kMlpBins : kMlpHidden;
        ERQ_CUDA(cudaMalloc(p, n * cols * 4));
        owned.push_back(*p);
    }
    ERQ_CUDA(cudaMalloc(&wk.xs, n * 2 * kMlpIn * sizeof(__nv_bfloat16)));
    owned.push_back(wk.xs);
    ERQ_CUDA(cudaMalloc(&wk.hs, n * 2 * kMlpHidden * sizeof(__nv_bfloat16)));
    owned.push_back(wk.hs);
    ERQ_TRY(mlp_infer(m, fin, wk, (int)n, pout, st));
    if (!p_dev) ERQ_CUDA(cudaMemcpyAsync(probs, pout, n * kMlpBins * 4, cudaMemcpyDeviceToHost, st));
    ERQ_CUDA(cudaStreamSynchronize(st));
    return ERQ_OK;
}

static erq_status search_learned_entry(const erq_index* idx, const erq_probe_model* m,
                                       const float* queries, bool rotated, uint64_t nq,
                                       uint64_t k, uint64_t nprobe_fallback, float confidence,
                                       float min_prob, uint32_t* ids, float* dists,
                                       uint32_t* nprobe_used, void* stream) {
    if (!m) return fail(ERQ_ERR_INVALID_ARGUMENT, "model is NULL");
    const float* rotated_queries = queries;
    ERQ_TRY(check_search_args(idx, nq, k, nprobe_fallback, queries, ids));
    if (idx->factors != 1)
        return fail(ERQ_ERR_UNSUPPORTED,
                    "learned probing takes indexes in the HIGH_ACC_FAST_SCAN format (one block factor)");
    if (nq == 0) return ERQ_OK;
    if (m->device != idx->device)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "model and index are on different devices");
    if (!(confidence > 0.f && confidence <= 1.f))
        return fail(ERQ_ERR_INVALID_ARGUMENT, "confidence must be in (0, 1]");
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint64_t nprobe_max =
        std::min<uint64_t>(idx->K, std::max<uint64_t>(nprobe_fallback, (uint64_t)m->bins[kMlpBins - 1]));
    ERQ_TRY(configure_kernels((int)idx->D, (int)idx->K, (int)k));
    const bool q_dev = is_device_ptr(rotated_queries), ids_dev = is_device_ptr(ids);
    const bool d_dev = dists == nullptr || is_device_ptr(dists);
    const bool u_dev = nprobe_used == nullptr || is_device_ptr(nprobe_used);
    Scratch s(st, idx->pool);
    const uint64_t in_cols = rotated ? idx->D : idx->DIM;
    const float* q = rotated_queries;
    if (!q_dev || (reinterpret_cast<uintptr_t>(q) & 15)) {
        float* tmp = nullptr;
        ERQ_TRY(s.alloc(&tmp, nq * in_cols));
        ERQ_CUDA(cudaMemcpyAsync(tmp, rotated_queries, nq * in_cols * 4, cudaMemcpyDefault, st));
        q = tmp;
    }
    if (!rotated) {
        float* tmp = nullptr;
        ERQ_TRY(s.alloc(&tmp, nq * idx->D));
        ERQ_TRY(rotate_device(idx, q, nq, tmp, st));
        q = tmp;
    }
    uint32_t* ids_out = ids;
    float* d_out = dists;
    int* used = nullptr;
    if (!ids_dev) ERQ_TRY(s.alloc(&ids_out, nq * k));
    if (!d_dev) ERQ_TRY(s.alloc(&d_out, nq * k));
    ERQ_TRY(s.alloc(&used, nq));
    const uint64_t bq = batch_queries(idx, nprobe_max, nq);
    Batch b;
    ERQ_TRY(alloc_batch(s, idx, bq, nprobe_max, b));
    ERQ_TRY(alloc_probe_lists(s, bq, b));
    float *near_d = nullptr, *feats = nullptr;
    ERQ_TRY(s.alloc(&near_d, bq * kFeatDists));
    ERQ_TRY(s.alloc(&feats, bq * kMlpIn));
    MlpWork wk;
    ERQ_TRY(mlp_alloc(s, (int)bq, false, wk));
    for (uint64_t q0 = 0; q0 < nq; q0 += bq) {
        b.nq = std::min(bq, nq - q0);
        b.qrot = q + q0 * idx->D;
        const int B = (int)b.nq;
        bool split = false;
        ERQ_TRY(features_device(idx, b, nprobe_max, near_d, feats, st, m, wk.xs, &split));
        ERQ_TRY(mlp_infer(m, feats, wk, B, wk.probs, st, true));
        {
            LaunchTimer t(kMlp, st);
            mlp_choose_nprobe_kernel<<<(unsigned)div_up(B, 128), 128, 0, st>>>(
                wk.probs, B, m->bins_dev, confidence, min_prob, (int)nprobe_fallback, (int)nprobe_max,
                used + q0);
            t.finish();
        }
        ERQ_CUDA(cudaGetLastError());
        // exact distances only as deep as each query's chosen depth
        if (split) ERQ_TRY(launch_probe_finish(idx, b, nprobe_max, st, used + q0));
        erq_status oe;
        const bool ordered = launch_order(idx, b, nprobe_max, st, used + q0, &oe);
        ERQ_TRY(oe);
        ERQ_TRY(launch_scan(idx, b, nprobe_max, st, used + q0, ordered ? b.order_pairs : nullptr));
        ERQ_TRY(launch_refine(idx, b, nprobe_max, k, ids_out + q0 * k,
                              d_out ? d_out + q0 * k : nullptr, st, used + q0,
                              ordered ? b.order_q : nullptr));
    }
    if (nprobe_used)
        ERQ_CUDA(cudaMemcpyAsync(nprobe_used, used, nq * 4, cudaMemcpyDefault, st));
    if (!ids_dev)
        ERQ_CUDA(cudaMemcpyAsync(ids, ids_out, nq * k * 4, cudaMemcpyDeviceToHost, st));
    if (!d_dev)
        ERQ_CUDA(cudaMemcpyAsync(dists, d_out, nq * k * 4, cudaMemcpyDeviceToHost, st));
    if (!q_dev || !ids_dev || !d_dev || !u_dev) {
        uint32_t* hw = nullptr;
        ERQ_TRY(tc_status_fetch(st, &hw));
        ERQ_CUDA(cudaStreamSynchronize(st));
        ERQ_TRY(tc_status_check(hw));
    }
    return ERQ_OK;
}

erq_status erq_search_learned(const erq_index* idx, const erq_probe_model* m,
                              const float* rotated_queries, uint64_t nq, uint64_t k,
                              uint64_t nprobe_fallback, float confidence, float min_prob,
                              uint32_t* ids, float* dists, uint32_t* nprobe_used, void* stream) {
    return search_learned_entry(idx, m, rotated_queries, true, nq, k, nprobe_fallback, confidence,
                                min_prob, ids, dists, nprobe_used, stream);
}

erq_status erq_search_learned_raw(const erq_index* idx, const erq_probe_model* m,
                                  const float* queries, uint64_t nq, uint64_t k,
                                  uint64_t nprobe_fallback, float confidence, float min_prob,
                                  uint32_t* ids, float* dists, uint32_t* nprobe_used,
                                  void* stream) {
    return search_learned_entry(idx, m, queries, false, nq, k, nprobe_fallback, confidence,
                                min_prob, ids, dists, nprobe_used, stream);
}

erq_status erq_debug_probe_model_grads(const erq_probe_model* m, const float* features,
                                       const uint8_t* labels, uint64_t n, float* loss,
                                       float* grads) {
    if (!m || !features || !labels || !loss || !grads)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0 || n > 65536) return fail(ERQ_ERR_INVALID_ARGUMENT, "n must be in [1, 65536]");
    DeviceGuard guard;
    ERQ_TRY(guard.set(m->device));
    std::vector<void*> owned;
    struct Frees {
        std::vector<void*>& p;
        ~Frees() {
            for (void* x : p) cudaFree(x);
        }
    } frees{owned};
    auto dm = [&](void** p, size_t bytes) -> erq_status {
        ERQ_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 16)));
        owned.push_back(*p);
        return ERQ_OK;
    };
    float *fin = nullptr, *g = nullptr;
    uint8_t* y = nullptr;
    MlpWork wk;
    ERQ_TRY(dm((void**)&fin, n * kMlpIn * 4));
    ERQ_TRY(dm((void**)&y, n));
    ERQ_TRY(dm((void**)&g, kMlpParams * 4));
    ERQ_TRY(dm((void**)&wk.x, n * kMlpIn * 4));
    ERQ_TRY(dm((void**)&wk.h1, n * kMlpHidden * 4));
    ERQ_TRY(dm((void**)&wk.h2, n * kMlpHidden * 4));
    ERQ_TRY(dm((void**)&wk.z, n * kMlpBins * 4));
    ERQ_TRY(dm((void**)&wk.probs, n * kMlpBins * 4));
    ERQ_TRY(dm((void**)&wk.dz, n * kMlpBins * 4));
    ERQ_TRY(dm((void**)&wk.dh2, n * kMlpHidden * 4));
    ERQ_TRY(dm((void**)&wk.dh1, n * kMlpHidden * 4));
    ERQ_TRY(dm((void**)&wk.loss, n * 4));
    ERQ_CUDA(cudaMemcpy(fin, features, n * kMlpIn * 4, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(y, labels, n, cudaMemcpyHostToDevice));
    cudaStream_t st = nullptr;
    mlp_standardise_kernel<<<(unsigned)div_up(n * kMlpIn, 256), 256, 0, st>>>(fin, m->mean, m->stdv,
                                                                            wk.x, (int)(n * kMlpIn));
    ERQ_TRY(mlp_forward(m, wk, (int)n, st));
    mlp_softmax_xent_kernel<<<(unsigned)div_up(n, 128), 128, 0, st>>>(wk.z, y, (int)n, wk.probs, wk.dz,
                                                                     wk.loss);
    ERQ_TRY(mlp_backward(m, wk, (int)n, g, st));
    std::vector<float> lh(n);
    ERQ_CUDA(cudaMemcpy(lh.data(), wk.loss, n * 4, cudaMemcpyDeviceToHost));
    ERQ_CUDA(cudaMemcpy(grads, g, kMlpParams * 4, cudaMemcpyDeviceToHost));
    double sum = 0.0;
    for (float v : lh) sum += v;
    *loss = (float)(sum / n);
    return ERQ_OK;
}

erq_status erq_debug_probe_model_params(const erq_probe_model* m, float* params, float* mean,
                                        float* stdv, uint32_t* bin_nprobe) {
    if (!m) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard guard;
    ERQ_TRY(guard.set(m->device));
    if (params) ERQ_CUDA(cudaMemcpy(params, m->w, kMlpParams * 4, cudaMemcpyDeviceToHost));
    if (mean) ERQ_CUDA(cudaMemcpy(mean, m->mean, kMlpIn * 4, cudaMemcpyDeviceToHost));
    if (stdv) ERQ_CUDA(cudaMemcpy(stdv, m->stdv, kMlpIn * 4, cudaMemcpyDeviceToHost));
    if (bin_nprobe)
        for (int j = 0; j < kMlpBins; ++j) bin_nprobe[j] = (uint32_t)m->bins[j];
    return ERQ_OK;
}

void erq_profile_enable(int on) {
    Profiler& p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    p.on = on != 0;
}

void erq_profile_reset(void) {
    Profiler& p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    for (auto& r : p.pending) {
        cudaEventSynchronize(r.stop);
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    p.pending.clear();
    for (int i = 0; i < kNumKernels; ++i) {
        p.launches[i] = 0;
        p.ms[i] = 0.0;
    }
}

erq_status erq_debug_gemm_bf16(const uint16_t* A, const uint16_t* B, uint64_t M, uint64_t N,
                               uint64_t Kd, float* C, int device) {
    if (!A || !B || !C) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (M == 0 || N == 0 || Kd == 0 || M > (1u << 30) || N > (1u << 30) || Kd > (1u << 20))
        return fail(ERQ_ERR_INVALID_ARGUMENT, "bad GEMM shape");
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    std::vector<void*> owned;
    struct Free {
        std::vector<void*>& v;
        ~Free() {
            for (void* p : v) cudaFree(p);
        }
    } frees{owned};
    __nv_bfloat16 *a = nullptr, *b = nullptr;
    float* c = nullptr;
    ERQ_CUDA(cudaMalloc(&a, M * Kd * 2));
    owned.push_back(a);
    ERQ_CUDA(cudaMalloc(&b, N * Kd * 2));
    owned.push_back(b);
    ERQ_CUDA(cudaMalloc(&c, M * N * 4));
    owned.push_back(c);
    ERQ_CUDA(cudaMemcpy(a, A, M * Kd * 2, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(b, B, N * Kd * 2, cudaMemcpyHostToDevice));
    uint32_t* status = nullptr;
    ERQ_TRY(tc_status_ptr(&status));
    ERQ_CUDA(cudaMemset(status, 0, 4));
    ERQ_TRY(gemm_tc(a, b, c, (int)M, (int)N, (int)Kd, GemmEpilogue(), kGemm, nullptr));
    ERQ_CUDA(cudaDeviceSynchronize());
    uint32_t st = 0;
    ERQ_CUDA(cudaMemcpy(&st, status, 4, cudaMemcpyDeviceToHost));
    if (st) return fail(ERQ_ERR_TIMEOUT, "a wait in the tcgen05 GEMM reached its limit");
    ERQ_CUDA(cudaMemcpy(C, c, M * N * 4, cudaMemcpyDeviceToHost));
    return ERQ_OK;
}

erq_status erq_build_index(const float* data, uint64_t n, uint64_t dim, const float* centroids,
                           uint64_t k, const uint32_t* cluster_ids, uint64_t total_bits,
                           const float* rotation, uint64_t seed, const char* path, int device) {
    if (!data || !centroids || !cluster_ids || !path)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint64_t EX = total_bits - 1;
    if (total_bits < 3 || !(EX == 2 || EX == 3 || EX == 4 || EX == 6 || EX == 7 || EX == 8))
        return fail(ERQ_ERR_INVALID_ARGUMENT, "total_bits=%llu: 3, 4, 5, 7, 8 or 9 expected",
                    (unsigned long long)total_bits);
    const uint64_t D = (dim + 63) / 64 * 64;
    if (n == 0 || dim == 0 || k == 0 || D > (uint64_t)kMaxD || n >= (1ull << 31) || k > kMaxClusters)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "bad shape (n=%llu dim=%llu k=%llu)",
                    (unsigned long long)n, (unsigned long long)dim, (unsigned long long)k);
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    // file order: clusters in order, members by ascending data index
    std::vector<uint32_t> cid_h(n);
    ERQ_CUDA(cudaMemcpy(cid_h.data(), cluster_ids, n * sizeof(uint32_t), cudaMemcpyDefault));
    std::vector<uint64_t> sizes(k, 0);
    for (uint64_t i = 0; i < n; ++i) {
        if (cid_h[i] >= k) return fail(ERQ_ERR_INVALID_ARGUMENT, "cluster id %u >= k", cid_h[i]);
        ++sizes[cid_h[i]];
    }
    std::vector<uint64_t> first(k + 1, 0);
    for (uint64_t c = 0; c < k; ++c) first[c + 1] = first[c] + sizes[c];
    std::vector<uint32_t> order(n), cid_row(n);
    {
        std::vector<uint64_t> pos(first.begin(), first.end() - 1);
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t p = pos[cid_h[i]]++;
            order[p] = (uint32_t)i;
            cid_row[p] = cid_h[i];
        }
    }
    std::vector<uint32_t> vfirst, vnum;
    for (uint64_t c = 0; c < k; ++c)
        for (uint64_t b = 0; b < sizes[c]; b += 32) {
            vfirst.push_back((uint32_t)(first[c] + b));
            vnum.push_back((uint32_t)std::min<uint64_t>(32, sizes[c] - b));
        }
    const uint64_t nblocks = vfirst.size();
    // rotation: the caller's D x D matrix, else a seeded random orthogonal one
    std::vector<float> P(D * D);
    if (rotation) {
        ERQ_CUDA(cudaMemcpy(P.data(), rotation, D * D * sizeof(float), cudaMemcpyDefault));
    } else {
        random_rotation(D, seed, P);
    }
    KmBuffers b;
    float *x = nullptr, *cent = nullptr, *Pd = nullptr, *cp = nullptr, *xp = nullptr, *onorm = nullptr,
          *ipn = nullptr, *xip = nullptr;
    uint32_t *ord = nullptr, *cidr = nullptr, *vf = nullptr, *vn = nullptr;
    uint64_t* bits = nullptr;
    uint8_t *code = nullptr, *lng = nullptr, *shrt = nullptr;
    const uint64_t lrow = D * EX / 8, bb = 4 * D + 128;
    ERQ_TRY(b.alloc(&x, n * dim));
    ERQ_TRY(b.alloc(&cent, k * dim));
    ERQ_TRY(b.alloc(&Pd, D * D));
    ERQ_TRY(b.alloc(&cp, k * D));
    ERQ_TRY(b.alloc(&xp, n * D));
    ERQ_TRY(b.alloc(&onorm, n));
    ERQ_TRY(b.alloc(&ipn, n));
    ERQ_TRY(b.alloc(&xip, n));
    ERQ_TRY(b.alloc(&ord, n));
    ERQ_TRY(b.alloc(&cidr, n));
    ERQ_TRY(b.alloc(&vf, std::max<uint64_t>(nblocks, 1)));
    ERQ_TRY(b.alloc(&vn, std::max<uint64_t>(nblocks, 1)));
    ERQ_TRY(b.alloc(&bits, n * (D / 64)));
    ERQ_TRY(b.alloc(&code, n * D));
    ERQ_TRY(b.alloc(&lng, n * lrow));
    ERQ_TRY(b.alloc(&shrt, std::max<uint64_t>(nblocks, 1) * bb));
    ERQ_CUDA(cudaMemcpy(x, data, n * dim * sizeof(float), cudaMemcpyDefault));
    ERQ_CUDA(cudaMemcpy(cent, centroids, k * dim * sizeof(float), cudaMemcpyDefault));
    ERQ_CUDA(cudaMemcpy(Pd, P.data(), D * D * sizeof(float), cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(ord, order.data(), n * 4, cudaMemcpyHostToDevice));
    ERQ_CUDA(cudaMemcpy(cidr, cid_row.data(), n * 4, cudaMemcpyHostToDevice));
    if (nblocks) {
        ERQ_CUDA(cudaMemcpy(vf, vfirst.data(), nblocks * 4, cudaMemcpyHostToDevice));
        ERQ_CUDA(cudaMemcpy(vn, vnum.data(), nblocks * 4, cudaMemcpyHostToDevice));
    }
    {
        dim3 gc((unsigned)div_up(D, kBuildBN), (unsigned)div_up(k, kBuildBM));
        build_rotate_kernel<<<gc, 256>>>(cent, (int)dim, nullptr, (int)k, Pd, (int)D, nullptr, nullptr, cp);
        ERQ_CUDA(cudaGetLastError());
        for (uint64_t r0 = 0; r0 < n; r0 += 65535ull * kBuildBM) {
            const uint64_t rows = std::min<uint64_t>(n - r0, 65535ull * kBuildBM);
            dim3 gx((unsigned)div_up(D, kBuildBN), (unsigned)div_up(rows, kBuildBM));
            build_rotate_kernel<<<gx, 256>>>(x, (int)dim, ord + r0, (int)rows, Pd, (int)D, cp, cidr + r0,
                                             xp + r0 * D);
            ERQ_CUDA(cudaGetLastError());
        }
    }
    build_x2_kernel<<<(unsigned)div_up(n * 16, 256), 256>>>(x, ord, cent, cidr, (int)n, (int)dim, onorm);
    ERQ_CUDA(cudaGetLastError());
    build_rows_kernel<<<(unsigned)div_up(n, 128), 128>>>(xp, (int)n, (int)D, bits);
    ERQ_CUDA(cudaGetLastError());
    {
        const uint64_t T = std::min<uint64_t>(n, 65536);
        double* ht = nullptr;
        uint16_t* hi = nullptr;
        uint8_t* cur = nullptr;
        ERQ_TRY(b.alloc(&ht, T * D));
        ERQ_TRY(b.alloc(&hi, T * D));
        ERQ_TRY(b.alloc(&cur, T * D));
        for (uint64_t r0 = 0; r0 < n; r0 += T) {
            fast_quantize_kernel<<<(unsigned)div_up(T, 128), 128>>>(xp, (int)n, (int)r0, (int)T, (int)D,
                                                                    (int)EX, ht, hi, cur, code, ipn);
            ERQ_CUDA(cudaGetLastError());
        }
    }
    build_long_kernel<<<(unsigned)div_up(n * (D / 64), 128), 128>>>(code, bits, ipn, onorm, (int)n, (int)D,
                                                                    (int)EX, lng, xip);
    ERQ_CUDA(cudaGetLastError());
    if (nblocks) {
        build_short_kernel<<<2368, 256>>>(bits, onorm, vf, vn, nblocks, (int)D, shrt);
        ERQ_CUDA(cudaGetLastError());
    }
    ERQ_CUDA(cudaDeviceSynchronize());
    // IVF::save (inc/index/IVF.hpp:219-252)
    std::unique_ptr<FILE, FileCloser> f(fopen(path, "wb"));
    if (!f) return fail(ERQ_ERR_IO, "cannot create '%s'", path);
    auto put = [&](const void* p, size_t bytes) -> erq_status {
        if (bytes && fwrite(p, 1, bytes, f.get()) != bytes) return fail(ERQ_ERR_IO, "write to '%s' failed", path);
        return ERQ_OK;
    };
    auto put_dev = [&](const void* dptr, size_t bytes) -> erq_status {
        std::vector<uint8_t> h(std::min<size_t>(bytes, 256ull << 20));
        for (size_t off = 0; off < bytes; off += h.size()) {
            const size_t m = std::min(h.size(), bytes - off);
            ERQ_CUDA(cudaMemcpy(h.data(), static_cast<const uint8_t*>(dptr) + off, m, cudaMemcpyDeviceToHost));
            ERQ_TRY(put(h.data(), m));
        }
        return ERQ_OK;
    };
    const uint64_t hdr[4] = {n, dim, k, EX};
    ERQ_TRY(put(hdr, sizeof(hdr)));
    ERQ_TRY(put(sizes.data(), k * sizeof(uint64_t)));
    ERQ_TRY(put(P.data(), D * D * sizeof(float)));
    ERQ_TRY(put_dev(cp, k * D * sizeof(float)));
    ERQ_TRY(put_dev(shrt, nblocks * bb));
    ERQ_TRY(put_dev(lng, n * lrow));
    ERQ_TRY(put_dev(xip, n * sizeof(float)));
    ERQ_TRY(put(order.data(), n * sizeof(uint32_t)));
    if (fflush(f.get()) != 0) return fail(ERQ_ERR_IO, "write to '%s' failed", path);
    return ERQ_OK;
}

erq_status erq_kmeans(const float* data, uint64_t n, uint64_t dim, uint64_t k, int iters,
                      uint64_t seed, float* centroids, uint32_t* assign, int device) {
    if (!data || !centroids) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0 || dim == 0 || k == 0 || k > n || iters < 0 || n > 0x7fffffffull ||
        dim > (uint64_t)kMaxD * 8 || k > 0x7fffffffull)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "bad k-means shape (n=%llu dim=%llu k=%llu)",
                    (unsigned long long)n, (unsigned long long)dim, (unsigned long long)k);
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    cudaStream_t st = nullptr;
    KmBuffers b;
    const float* x = data;
    if (!is_device_ptr(data)) {
        float* xd = nullptr;
        ERQ_TRY(b.alloc(&xd, n * dim));
        ERQ_CUDA(cudaMemcpy(xd, data, n * dim * sizeof(float), cudaMemcpyHostToDevice));
        x = xd;
    }
    float* cent = nullptr;
    uint32_t* asg = nullptr;
    uint64_t* rows = nullptr;
    ERQ_TRY(b.alloc(&cent, k * dim));
    ERQ_TRY(b.alloc(&asg, n));
    ERQ_TRY(b.alloc(&rows, k));
    // initial centroids: k distinct points (partial Fisher-Yates shuffle)
    uint64_t rng = seed;
    {
        std::vector<uint64_t> perm(n);
        std::iota(perm.begin(), perm.end(), 0ull);
        for (uint64_t i = 0; i < k; ++i) std::swap(perm[i], perm[i + splitmix64_next(rng) % (n - i)]);
        ERQ_CUDA(cudaMemcpy(rows, perm.data(), k * sizeof(uint64_t), cudaMemcpyHostToDevice));
    }
    gather_rows_kernel<<<1184, 256, 0, st>>>(x, (int)dim, rows, (int)k, cent);
    ERQ_CUDA(cudaGetLastError());
    ERQ_TRY(km_iterate(x, n, dim, k, iters, cent, asg, rng, nullptr, true, st));
    ERQ_CUDA(cudaMemcpy(centroids, cent, k * dim * sizeof(float), cudaMemcpyDefault));
    if (assign) ERQ_CUDA(cudaMemcpy(assign, asg, n * sizeof(uint32_t), cudaMemcpyDefault));
    return ERQ_OK;
}

erq_status erq_kmeans_step(const float* data, uint64_t n, uint64_t dim, uint64_t k,
                           const float* centroids_in, uint64_t seed, float* centroids_out,
                           uint32_t* assign, uint32_t* counts, int device) {
    if (!data || !centroids_in || !centroids_out || !assign || !counts)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0 || dim == 0 || k == 0 || n > 0x7fffffffull || dim > (uint64_t)kMaxD * 8 ||
        k > 0x7fffffffull)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "bad k-means shape");
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    cudaStream_t st = nullptr;
    KmBuffers b;
    const float* x = data;
    if (!is_device_ptr(data)) {
        float* xd = nullptr;
        ERQ_TRY(b.alloc(&xd, n * dim));
        ERQ_CUDA(cudaMemcpy(xd, data, n * dim * sizeof(float), cudaMemcpyHostToDevice));
        x = xd;
    }
    float* cent = nullptr;
    uint32_t* asg = nullptr;
    ERQ_TRY(b.alloc(&cent, k * dim));
    ERQ_TRY(b.alloc(&asg, n));
    ERQ_CUDA(cudaMemcpy(cent, centroids_in, k * dim * sizeof(float), cudaMemcpyDefault));
    uint64_t rng = seed;
    std::vector<uint32_t> cnt(k);
    ERQ_TRY(km_iterate(x, n, dim, k, 1, cent, asg, rng, cnt.data(), false, st));
    ERQ_CUDA(cudaMemcpy(centroids_out, cent, k * dim * sizeof(float), cudaMemcpyDefault));
    ERQ_CUDA(cudaMemcpy(assign, asg, n * sizeof(uint32_t), cudaMemcpyDefault));
    ERQ_CUDA(cudaMemcpy(counts, cnt.data(), k * sizeof(uint32_t), cudaMemcpyDefault));
    return ERQ_OK;
}

erq_status erq_debug_set_gemm_wait_limit(uint32_t polls) {
    g_tc_wait_limit.store(polls ? polls : kTcWaitLimit);
    return ERQ_OK;
}

erq_status erq_debug_probe_fallbacks(int device, uint64_t* count, int reset) {
    if (!count) return fail(ERQ_ERR_INVALID_ARGUMENT, "count is NULL");
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    uint32_t* c = probe_fallback_counter();
    if (!c) return fail(ERQ_ERR_CUDA, "fallback counter unavailable");
    uint32_t v = 0;
    ERQ_CUDA(cudaMemcpy(&v, c, sizeof(v), cudaMemcpyDeviceToHost));
    *count = v;
    if (reset) ERQ_CUDA(cudaMemset(c, 0, sizeof(uint32_t)));
    return ERQ_OK;
}

erq_status erq_debug_refine_stats(int device, int enable, uint64_t stats[4]) {
    if (!stats) return fail(ERQ_ERR_INVALID_ARGUMENT, "stats is NULL");
    DeviceGuard guard;
    ERQ_TRY(guard.set(device));
    unsigned long long* c = refine_stats_counter();
    if (!c) return fail(ERQ_ERR_CUDA, "refinement counters unavailable");
    ERQ_CUDA(cudaDeviceSynchronize());
    unsigned long long v[4] = {};
    ERQ_CUDA(cudaMemcpy(v, c, sizeof(v), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 4; ++i) stats[i] = v[i];
    ERQ_CUDA(cudaMemset(c, 0, sizeof(v)));
    g_refine_stats_on.store(enable != 0);
    return ERQ_OK;
}

erq_status erq_profile_read(const char* kernel, uint64_t* launches, double* total_ms) {
    if (!kernel || !launches || !total_ms) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    int id = -1;
    for (int i = 0; i < kNumKernels; ++i)
        if (strcmp(kernel, kKernelNames[i]) == 0) id = i;
    if (id < 0) return fail(ERQ_ERR_INVALID_ARGUMENT, "unknown kernel '%s'", kernel);
    Profiler& p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    for (auto& r : p.pending) {
        ERQ_CUDA(cudaEventSynchronize(r.stop));
        float ms = 0.f;
        ERQ_CUDA(cudaEventElapsedTime(&ms, r.start, r.stop));
        p.launches[r.kernel] += 1;
        p.ms[r.kernel] += ms;
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    p.pending.clear();
    *launches = p.launches[id];
    *total_ms = p.ms[id];
    return ERQ_OK;
}

}  // extern "C"

// ------------------------------------------------------------ batched plans
//
// A plan holds every buffer a search of up to max_batch queries needs, so a
// search allocates nothing; the whole pipeline of one batch size is captured
// once into a CUDA graph and replayed.  The scan runs over the
// (query block x cluster chunk) work list of scan_batch.cuh with tiles the
// autotuner picks.
namespace {

struct Arena {
    std::vector<void*> ptrs;
    uint64_t bytes = 0;
    template <typename T>
    erq_status alloc(T** out, size_t count) {
        void* p = nullptr;
        const size_t b = std::max<size_t>(count * sizeof(T), 16);
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? ERQ_ERR_OUT_OF_MEMORY : ERQ_ERR_CUDA,
                        "cudaMalloc(%zu bytes) for a plan failed: %s", b, cudaGetErrorString(e));
        ptrs.push_back(p);
        bytes += b;
        *out = static_cast<T*>(p);
        return ERQ_OK;
    }
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
};

// Scan tile shapes the autotuner chooses among: (queries per item, warps).
struct ScanShape {
    int qb, warps;
};
constexpr ScanShape kScanShapes[] = {{1, 4}, {1, 8}, {2, 4}, {2, 8}, {4, 4}, {4, 8}};
constexpr int kNumScanShapes = sizeof(kScanShapes) / sizeof(kScanShapes[0]);
constexpr int kChunkChoices[] = {8, 16, 32, 64};

// Calls f with the kernel instantiation for (QB, W) and D's table stride
// class (one instantiation serves every D when QB = 1).
template <int QB, int W, typename F>
erq_status with_scan_batched(int D, F&& f) {
    if constexpr (QB == 1) {
        return f(scan_batched_kernel<1, W, 0>, scan_batch_smem_bytes(1, W, 0, D));
    } else {
        switch (scan_qstride(D)) {
            case 16384:
                return f(scan_batched_kernel<QB, W, 16384>, scan_batch_smem_bytes(QB, W, 16384, D));
            case 32768:
                return f(scan_batched_kernel<QB, W, 32768>, scan_batch_smem_bytes(QB, W, 32768, D));
            default:
                return f(scan_batched_kernel<QB, W, 45056>, scan_batch_smem_bytes(QB, W, 45056, D));
        }
    }
}

// Resident blocks per SM of shape (QB, W) at this D; 0 when its shared
// memory exceeds what a block may have (the shape is then never used).
template <int QB, int W>
erq_status scan_batched_configure(int D, int* per_sm) {
    *per_sm = 0;
    int dev = 0, optin = 0;
    ERQ_CUDA(cudaGetDevice(&dev));
    ERQ_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    return with_scan_batched<QB, W>(D, [&](auto kern, size_t smem) -> erq_status {
        if (smem > (size_t)optin) return ERQ_OK;
        ERQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ERQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, W * 32, smem));
        return ERQ_OK;
    });
}

template <int QB, int W>
erq_status scan_batched_launch(const ScanBatchArgs& a, int blocks, cudaStream_t st) {
    if (blocks <= 0)
        return fail(ERQ_ERR_UNSUPPORTED, "scan tile (%d queries, %d warps) does not fit at D=%d", QB,
                    W, a.D);
    return with_scan_batched<QB, W>(a.D, [&](auto kern, size_t smem) -> erq_status {
        LaunchTimer t(kScan, st);
        kern<<<(unsigned)blocks, W * 32, smem, st>>>(a);
        t.finish();
        ERQ_CUDA(cudaGetLastError());
        return ERQ_OK;
    });
}

}  // namespace

struct erq_plan {
    const erq_index* idx = nullptr;
    const erq_probe_model* model = nullptr;
    uint64_t max_batch = 0, k = 0, nprobe = 0, nprobe_run = 0;
    bool raw = false;
    float confidence = 0.9f, min_prob = 0.f;
    int sms = 148;
    int per_sm[kNumScanShapes] = {};  // resident scan blocks per SM, by kScanShapes entry
    std::map<uint64_t, erq_plan_tuning> tunings;  // by the batch size tuned for
    Arena arena;
    Batch b;
    float* qin = nullptr;       // [max_batch][DIM or D] queries as given
    float* qrot = nullptr;      // [max_batch][D]
    uint32_t* ids = nullptr;    // [max_batch][k]
    float* dists = nullptr;     // [max_batch][k]
    int* used = nullptr;        // [max_batch] clusters probed per query
    float* near_d = nullptr;    // [max_batch][64]
    float* feats = nullptr;     // [max_batch][320]
    MlpWork wk;
    uint32_t* item_off = nullptr;  // [K + 1]
    uint32_t* counter = nullptr;
    cudaStream_t cap = nullptr;
    bool use_graphs = true;
    std::mutex mu;
    std::map<uint64_t, cudaGraphExec_t> graphs;  // by 2 * batch size + buffer slot
    // Host-buffer pipelining: a batch with host buffers runs as chunks; chunk
    // i uses buffer slot i % 2 (slot 0 = qin/ids/dists/used above, slot 1 =
    // the buffers below, slot_rows queries), so the copy of chunk i + 1's
    // queries in and chunk i - 1's results out overlap chunk i's search.
    uint64_t slot_rows = 0;  // 0: plan too small to pipeline
    float* qin1 = nullptr;
    uint32_t* ids1 = nullptr;
    float* dists1 = nullptr;
    int* used1 = nullptr;
    int pipe_chunks = 1;     // erq_plan_set_pipeline: 1 = one piece (default), 0 = by size
    int next_slot = 0;       // erq_plan_search_async: the slot of the next call
    bool slot_used[2] = {false, false};
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    cudaEvent_t ev_in[2] = {}, ev_comp[2] = {}, ev_out[2] = {};

    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second);
        graphs.clear();
    }
    ~erq_plan() {
        int prev = -1;
        cudaGetDevice(&prev);
        if (idx) cudaSetDevice(idx->device);
        cudaDeviceSynchronize();
        drop_graphs();
        if (cap) cudaStreamDestroy(cap);
        if (h2d) cudaStreamDestroy(h2d);
        if (d2h) cudaStreamDestroy(d2h);
        for (cudaEvent_t e : {ev_start, ev_end, ev_in[0], ev_in[1], ev_comp[0], ev_comp[1], ev_out[0],
                              ev_out[1]})
            if (e) cudaEventDestroy(e);
        if (prev >= 0) cudaSetDevice(prev);
    }
};

namespace {

erq_plan_tuning default_tuning(uint64_t nq) {
    erq_plan_tuning t{};
    t.queries_per_item = nq >= 1024 ? 4 : 1;
    t.blocks_per_item = 16;
    t.warps = nq >= 1024 ? 8 : 4;
    t.refine_warps = 0;
    return t;
}

// Tuning for a batch of nq: the one tuned for the nearest batch size (log
// scale), else the default.
erq_plan_tuning plan_tuning(const erq_plan* p, uint64_t nq) {
    if (p->tunings.empty()) return default_tuning(nq);
    double best = 1e300;
    erq_plan_tuning t = p->tunings.begin()->second;
    for (auto& kv : p->tunings) {
        const double d = std::fabs(std::log((double)kv.first) - std::log((double)std::max<uint64_t>(nq, 1)));
        if (d < best) {
            best = d;
            t = kv.second;
        }
    }
    return t;
}

bool tuning_valid(const erq_plan_tuning& t) {
    bool shape = false;
    for (auto& sh : kScanShapes) shape |= (int)t.queries_per_item == sh.qb && (int)t.warps == sh.warps;
    return shape && t.blocks_per_item >= 1 && t.blocks_per_item <= 4096 &&
           (t.refine_warps == 0 || t.refine_warps == 4 || t.refine_warps == (uint32_t)kWideWarps);
}

erq_status launch_scan_batched(erq_plan* p, uint64_t nq, const erq_plan_tuning& t, cudaStream_t st) {
    const erq_index* idx = p->idx;
    const int K = (int)idx->K;
    {
        LaunchTimer lt(kOrder, st);
        scan_items_count_kernel<<<(unsigned)div_up(K, 256), 256, 0, st>>>(
            p->b.buckets, idx->c_nblocks, idx->c_by_size, K, (int)t.queries_per_item,
            (int)t.blocks_per_item, p->item_off);
        lt.finish();
    }
    {
        LaunchTimer lt(kOrder, st);
        bucket_scan_kernel<<<1, kBucketScanThreads, 0, st>>>(p->item_off, p->item_off, (uint32_t)K + 1);
        lt.finish();
    }
    ERQ_CUDA(cudaMemsetAsync(p->counter, 0, sizeof(uint32_t), st));
    ScanBatchArgs a{};
    a.qrot = p->b.qrot;
    a.centroids = idx->centroids;
    a.probe_cid = p->b.probe_cid;
    a.probe_sqy = p->b.probe_sqy;
    a.codes = idx->codes;
    a.c_first_block = idx->c_first_block;
    a.c_nblocks = idx->c_nblocks;
    a.s_off = p->b.s_off;
    a.S = p->b.S;
    a.qp_delta = p->b.delta;
    a.qp_sumq = p->b.sumq;
    a.onorm = idx->onorm;
    a.c_size = idx->c_size;
    a.bmin = p->b.bmin;
    a.order_pairs = p->b.order_pairs;
    a.bucket_end = p->b.buckets;
    a.item_off = p->item_off;
    a.c_order = idx->c_by_size;
    a.item_counter = p->counter;
    a.K = K;
    a.D = (int)idx->D;
    a.nprobe = (int)p->nprobe_run;
    a.CB = (int)t.blocks_per_item;
    (void)nq;
    ERQ_TRY(tc_status_ptr(&a.status));
    const int qb = (int)t.queries_per_item, w = (int)t.warps;
    auto grid = [&](int i) { return p->sms * p->per_sm[i]; };
    if (qb == 1 && w == 4) return scan_batched_launch<1, 4>(a, grid(0), st);
    if (qb == 1 && w == 8) return scan_batched_launch<1, 8>(a, grid(1), st);
    if (qb == 2 && w == 4) return scan_batched_launch<2, 4>(a, grid(2), st);
    if (qb == 2 && w == 8) return scan_batched_launch<2, 8>(a, grid(3), st);
    if (qb == 4 && w == 4) return scan_batched_launch<4, 4>(a, grid(4), st);
    if (qb == 4 && w == 8) return scan_batched_launch<4, 8>(a, grid(5), st);
    return fail(ERQ_ERR_INVALID_ARGUMENT, "unsupported scan tile (%d queries, %d warps)", qb, w);
}

// The device work of one batch of nq queries already in p->qin.
erq_status plan_pipeline(erq_plan* p, uint64_t nq, const erq_plan_tuning& t, cudaStream_t st) {
    const erq_index* idx = p->idx;
    Batch& b = p->b;
    b.nq = nq;
    if (p->raw) {
        ERQ_TRY(rotate_into(idx, p->qin, nq, p->qrot, b.qsplit, st));
        b.qrot = p->qrot;
    } else {
        b.qrot = p->qin;
    }
    const int* qnp = nullptr;
    if (p->model) {
        const erq_probe_model* m = p->model;
        const int B = (int)nq;
        bool split = false;
        ERQ_TRY(features_device(idx, b, p->nprobe_run, p->near_d, p->feats, st, m, p->wk.xs, &split));
        ERQ_TRY(mlp_infer(m, p->feats, p->wk, B, p->wk.probs, st, true));
        {
            LaunchTimer lt(kMlp, st);
            mlp_choose_nprobe_kernel<<<(unsigned)div_up(B, 128), 128, 0, st>>>(
                p->wk.probs, B, m->bins_dev, p->confidence, p->min_prob, (int)p->nprobe,
                (int)p->nprobe_run, p->used);
            lt.finish();
        }
        ERQ_CUDA(cudaGetLastError());
        // exact distances only as deep as each query's chosen depth
        if (split) ERQ_TRY(launch_probe_finish(idx, b, p->nprobe_run, st, p->used));
        qnp = p->used;
    } else {
        ERQ_TRY(launch_probe_tc(idx, b, p->nprobe_run, st));
    }
    ERQ_TRY(order_both(idx, b, p->nprobe_run, st, qnp, false));
    ERQ_TRY(launch_scan_batched(p, nq, t, st));
    ERQ_TRY(launch_refine(idx, b, p->nprobe_run, p->k, p->ids, p->dists, st, qnp, b.order_q,
                          (int)t.refine_warps));
    return ERQ_OK;
}

// Points the plan's query and result buffers at slot 1 for its lifetime.
struct SlotSwap {
    erq_plan* p;
    float* q;
    uint32_t* i;
    float* d;
    int* u;
    SlotSwap(erq_plan* pl, int slot) : p(pl), q(pl->qin), i(pl->ids), d(pl->dists), u(pl->used) {
        if (slot) {
            p->qin = p->qin1;
            p->ids = p->ids1;
            p->dists = p->dists1;
            p->used = p->used1;
        }
    }
    ~SlotSwap() {
        p->qin = q;
        p->ids = i;
        p->dists = d;
        p->used = u;
    }
};

// Graph of the pipeline for batch size nq on buffer slot `slot`, captured on
// first use.
erq_status plan_graph(erq_plan* p, uint64_t nq, int slot, cudaGraphExec_t* out) {
    const uint64_t key = 2 * nq + (uint64_t)slot;
    auto it = p->graphs.find(key);
    if (it != p->graphs.end()) {
        *out = it->second;
        return ERQ_OK;
    }
    const erq_plan_tuning t = plan_tuning(p, nq);
    cudaGraph_t g = nullptr;
    SlotSwap sw(p, slot);
    ERQ_CUDA(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
    erq_status s = plan_pipeline(p, nq, t, p->cap);
    cudaError_t e = cudaStreamEndCapture(p->cap, &g);
    if (s != ERQ_OK) {
        if (g) cudaGraphDestroy(g);
        return s;
    }
    if (e != cudaSuccess) return fail(ERQ_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    cudaGraphExec_t ge = nullptr;
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(ERQ_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    p->graphs[key] = ge;
    *out = ge;
    return ERQ_OK;
}

// Search of nq queries on buffer slot `slot`, asynchronous on st (queries
// already staged in the slot).
erq_status plan_run(erq_plan* p, uint64_t nq, int slot, cudaStream_t st) {
    if (p->use_graphs) {
        cudaGraphExec_t ge = nullptr;
        ERQ_TRY(plan_graph(p, nq, slot, &ge));
        ERQ_CUDA(cudaGraphLaunch(ge, st));
        return ERQ_OK;
    }
    SlotSwap sw(p, slot);
    return plan_pipeline(p, nq, plan_tuning(p, nq), st);
}

// Chunks a batch of nq queries with host buffers runs as (1: no pipelining).
uint64_t plan_chunks(const erq_plan* p, uint64_t nq) {
    if (!p->slot_rows || p->pipe_chunks == 1) return 1;
    uint64_t c = p->pipe_chunks ? (uint64_t)p->pipe_chunks : (nq >= 8192 ? 4 : (nq >= 4096 ? 2 : 1));
    c = std::min<uint64_t>(c, nq);
    while (c > 1 && div_up(nq, c) > p->slot_rows) --c;  // a chunk must fit slot 1
    return c;
}

// Search with host buffers as `chunks` pipelined chunks: H2D copies on p->h2d,
// the searches on st, D2H copies on p->d2h; chunk i uses slot i % 2 once
// chunk i - 2 has left it.  Returns with the copies ordered before st's next
// work.
erq_status plan_search_pipelined(erq_plan* p, const float* queries, uint64_t nq, uint64_t chunks,
                                 uint32_t* ids, float* dists, uint32_t* nprobe_used,
                                 cudaStream_t st) {
    const uint64_t cols = p->raw ? p->idx->DIM : p->idx->D;
    const uint64_t step = div_up(nq, chunks);
    ERQ_CUDA(cudaEventRecord(p->ev_start, st));
    ERQ_CUDA(cudaStreamWaitEvent(p->h2d, p->ev_start, 0));
    ERQ_CUDA(cudaStreamWaitEvent(p->d2h, p->ev_start, 0));
    for (uint64_t c = 0, q0 = 0; q0 < nq; ++c, q0 += step) {
        const int slot = (int)(c & 1);
        const uint64_t n = std::min(step, nq - q0);
        float* qin = slot ? p->qin1 : p->qin;
        if (c >= 2) ERQ_CUDA(cudaStreamWaitEvent(p->h2d, p->ev_comp[slot], 0));
        ERQ_CUDA(cudaMemcpyAsync(qin, queries + q0 * cols, n * cols * sizeof(float),
                                 cudaMemcpyDefault, p->h2d));
        ERQ_CUDA(cudaEventRecord(p->ev_in[slot], p->h2d));
        ERQ_CUDA(cudaStreamWaitEvent(st, p->ev_in[slot], 0));
        if (c >= 2) ERQ_CUDA(cudaStreamWaitEvent(st, p->ev_out[slot], 0));
        ERQ_TRY(plan_run(p, n, slot, st));
        ERQ_CUDA(cudaEventRecord(p->ev_comp[slot], st));
        ERQ_CUDA(cudaStreamWaitEvent(p->d2h, p->ev_comp[slot], 0));
        ERQ_CUDA(cudaMemcpyAsync(ids + q0 * p->k, slot ? p->ids1 : p->ids,
                                 n * p->k * sizeof(uint32_t), cudaMemcpyDefault, p->d2h));
        if (dists)
            ERQ_CUDA(cudaMemcpyAsync(dists + q0 * p->k, slot ? p->dists1 : p->dists,
                                     n * p->k * sizeof(float), cudaMemcpyDefault, p->d2h));
        if (nprobe_used)
            ERQ_CUDA(cudaMemcpyAsync(nprobe_used + q0, slot ? p->used1 : p->used,
                                     n * sizeof(uint32_t), cudaMemcpyDefault, p->d2h));
        ERQ_CUDA(cudaEventRecord(p->ev_out[slot], p->d2h));
    }
    ERQ_CUDA(cudaEventRecord(p->ev_end, p->d2h));
    ERQ_CUDA(cudaStreamWaitEvent(st, p->ev_end, 0));
    ERQ_CUDA(cudaEventRecord(p->ev_end, p->h2d));
    ERQ_CUDA(cudaStreamWaitEvent(st, p->ev_end, 0));
    return ERQ_OK;
}

erq_status plan_stage_queries(erq_plan* p, const float* queries, uint64_t nq, cudaStream_t st) {
    const uint64_t cols = p->raw ? p->idx->DIM : p->idx->D;
    ERQ_CUDA(cudaMemcpyAsync(p->qin, queries, nq * cols * sizeof(float), cudaMemcpyDefault, st));
    return ERQ_OK;
}

}  // namespace

extern "C" {

erq_status erq_plan_create(const erq_index* idx, const erq_probe_model* model, uint64_t max_batch,
                           uint64_t k, uint64_t nprobe, int raw_queries, erq_plan** out) {
    if (!out) return fail(ERQ_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (!idx) return fail(ERQ_ERR_INVALID_ARGUMENT, "index is NULL");
    if (idx->factors != 1)
        return fail(ERQ_ERR_UNSUPPORTED,
                    "batched plans take indexes in the HIGH_ACC_FAST_SCAN format (one block factor)");
    if (max_batch == 0) return fail(ERQ_ERR_INVALID_ARGUMENT, "max_batch must be positive");
    if (k == 0 || k > (uint64_t)kMaxTopK)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "k=%llu outside 1..%d", (unsigned long long)k, kMaxTopK);
    if (nprobe == 0) return fail(ERQ_ERR_INVALID_ARGUMENT, "nprobe must be positive");
    if (model && model->device != idx->device)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "model and index live on different devices");
    DeviceGuard guard;
    ERQ_TRY(guard.set(idx->device));
    std::unique_ptr<erq_plan> p(new erq_plan());
    p->idx = idx;
    p->model = model;
    p->max_batch = max_batch;
    p->k = k;
    p->nprobe = std::min<uint64_t>(nprobe, idx->K);
    p->nprobe_run = model ? std::min<uint64_t>(idx->K, std::max<uint64_t>(p->nprobe, (uint64_t)model->bins[kMlpBins - 1]))
                          : p->nprobe;
    p->raw = raw_queries != 0;
    ERQ_CUDA(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, idx->device));
    ERQ_TRY(configure_kernels((int)idx->D, (int)idx->K, (int)k));
    {
        const int D = (int)idx->D;
        ERQ_TRY((scan_batched_configure<1, 4>(D, &p->per_sm[0])));
        ERQ_TRY((scan_batched_configure<1, 8>(D, &p->per_sm[1])));
        ERQ_TRY((scan_batched_configure<2, 4>(D, &p->per_sm[2])));
        ERQ_TRY((scan_batched_configure<2, 8>(D, &p->per_sm[3])));
        ERQ_TRY((scan_batched_configure<4, 4>(D, &p->per_sm[4])));
        ERQ_TRY((scan_batched_configure<4, 8>(D, &p->per_sm[5])));
    }
    ERQ_TRY(alloc_batch(p->arena, idx, max_batch, p->nprobe_run, p->b));
    if (model) ERQ_TRY(alloc_probe_lists(p->arena, max_batch, p->b));
    ERQ_TRY(p->arena.alloc(&p->qin, max_batch * (p->raw ? idx->DIM : idx->D)));
    ERQ_TRY(p->arena.alloc(&p->qrot, max_batch * idx->D));
    ERQ_TRY(p->arena.alloc(&p->ids, max_batch * k));
    ERQ_TRY(p->arena.alloc(&p->dists, max_batch * k));
    ERQ_TRY(p->arena.alloc(&p->used, max_batch));
    ERQ_TRY(p->arena.alloc(&p->item_off, idx->K + 1));
    ERQ_TRY(p->arena.alloc(&p->counter, 1));
    if (model) {
        ERQ_TRY(p->arena.alloc(&p->near_d, max_batch * kFeatDists));
        ERQ_TRY(p->arena.alloc(&p->feats, max_batch * kMlpIn));
        ERQ_TRY(mlp_alloc(p->arena, (int)max_batch, false, p->wk));
    }
    {
        std::vector<int> np(max_batch, (int)p->nprobe);
        ERQ_CUDA(cudaMemcpy(p->used, np.data(), max_batch * sizeof(int), cudaMemcpyHostToDevice));
    }
    ERQ_CUDA(cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking));
    {  // a second buffer slot for pipelined and asynchronous host-buffer searches
        p->slot_rows = max_batch;
        ERQ_TRY(p->arena.alloc(&p->qin1, p->slot_rows * (p->raw ? idx->DIM : idx->D)));
        ERQ_TRY(p->arena.alloc(&p->ids1, p->slot_rows * k));
        ERQ_TRY(p->arena.alloc(&p->dists1, p->slot_rows * k));
        ERQ_TRY(p->arena.alloc(&p->used1, p->slot_rows));
        std::vector<int> np(p->slot_rows, (int)p->nprobe);
        ERQ_CUDA(cudaMemcpy(p->used1, np.data(), p->slot_rows * sizeof(int), cudaMemcpyHostToDevice));
        ERQ_CUDA(cudaStreamCreateWithFlags(&p->h2d, cudaStreamNonBlocking));
        ERQ_CUDA(cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&p->ev_start, &p->ev_end, &p->ev_in[0], &p->ev_in[1], &p->ev_comp[0],
                               &p->ev_comp[1], &p->ev_out[0], &p->ev_out[1]})
            ERQ_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    *out = p.release();
    return ERQ_OK;
}

void erq_plan_free(erq_plan* plan) { delete plan; }

erq_status erq_plan_set_learned(erq_plan* p, float confidence, float min_prob) {
    if (!p) return fail(ERQ_ERR_INVALID_ARGUMENT, "plan is NULL");
    if (!p->model) return fail(ERQ_ERR_INVALID_ARGUMENT, "the plan has no probe model");
    if (!(confidence > 0.f && confidence <= 1.f))
        return fail(ERQ_ERR_INVALID_ARGUMENT, "confidence must be in (0, 1]");
    std::lock_guard<std::mutex> g(p->mu);
    DeviceGuard guard;
    ERQ_TRY(guard.set(p->idx->device));
    p->confidence = confidence;
    p->min_prob = min_prob;
    p->drop_graphs();
    return ERQ_OK;
}

erq_status erq_plan_set_tuning(erq_plan* p, uint64_t batch, const erq_plan_tuning* t) {
    if (!p || !t) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!tuning_valid(*t)) return fail(ERQ_ERR_INVALID_ARGUMENT, "unsupported tuning");
    std::lock_guard<std::mutex> g(p->mu);
    DeviceGuard guard;
    ERQ_TRY(guard.set(p->idx->device));
    p->tunings[std::max<uint64_t>(batch, 1)] = *t;
    p->drop_graphs();
    return ERQ_OK;
}

erq_status erq_plan_get_tuning(const erq_plan* p, uint64_t batch, erq_plan_tuning* t) {
    if (!p || !t) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    *t = plan_tuning(p, batch);
    return ERQ_OK;
}

erq_status erq_plan_autotune(erq_plan* p, const float* queries, uint64_t n, int reps,
                             erq_plan_tuning* chosen, float* best_ms) {
    if (!p || !queries) return fail(ERQ_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n == 0 || n > p->max_batch)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "sample of %llu queries outside 1..max_batch",
                    (unsigned long long)n);
    std::lock_guard<std::mutex> g(p->mu);
    DeviceGuard guard;
    ERQ_TRY(guard.set(p->idx->device));
    cudaStream_t st = p->cap;
    ERQ_TRY(plan_stage_queries(p, queries, n, st));
    cudaEvent_t e0, e1;
    ERQ_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(ERQ_ERR_CUDA, "cudaEventCreate failed");
    }
    float best = 1e30f;
    erq_plan_tuning bt = default_tuning(n);
    erq_status s = ERQ_OK;
    for (int si = 0; si < kNumScanShapes && s == ERQ_OK; ++si) {
        const ScanShape& sh = kScanShapes[si];
        if (!p->per_sm[si]) continue;  // does not fit at this D
        for (int cb : kChunkChoices) {
            erq_plan_tuning t = default_tuning(n);  // refinement form by batch size
            t.queries_per_item = (uint32_t)sh.qb;
            t.blocks_per_item = (uint32_t)cb;
            t.warps = (uint32_t)sh.warps;
            if ((s = plan_pipeline(p, n, t, st)) != ERQ_OK) break;  // warm-up
            float ms = 1e30f;
            for (int r = 0; r < std::max(1, reps); ++r) {
                cudaEventRecord(e0, st);
                if ((s = plan_pipeline(p, n, t, st)) != ERQ_OK) break;
                cudaEventRecord(e1, st);
                cudaEventSynchronize(e1);
                float x = 0.f;
                cudaEventElapsedTime(&x, e0, e1);
                ms = std::min(ms, x);
            }
            if (s != ERQ_OK) break;
            if (ms < best) {
                best = ms;
                bt = t;
            }
        }
        if (s != ERQ_OK) break;
    }
    // both refinement forms with the chosen tile (the auto choice is one of them)
    for (uint32_t rw : {4u, (uint32_t)kWideWarps}) {
        if (s != ERQ_OK) break;
        erq_plan_tuning t = bt;
        t.refine_warps = rw;
        if ((s = plan_pipeline(p, n, t, st)) != ERQ_OK) break;  // warm-up
        float ms = 1e30f;
        for (int r = 0; r < std::max(1, reps); ++r) {
            cudaEventRecord(e0, st);
            if ((s = plan_pipeline(p, n, t, st)) != ERQ_OK) break;
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float x = 0.f;
            cudaEventElapsedTime(&x, e0, e1);
            ms = std::min(ms, x);
        }
        if (s == ERQ_OK && ms < best) {
            best = ms;
            bt = t;
        }
    }
    if (bt.refine_warps == 0) bt.refine_warps = n <= (uint64_t)device_sms() ? kWideWarps : 4;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ERQ_TRY(s);
    ERQ_CUDA(cudaStreamSynchronize(st));
    p->tunings[n] = bt;
    p->drop_graphs();
    if (chosen) *chosen = bt;
    if (best_ms) *best_ms = best;
    return ERQ_OK;
}

erq_status erq_plan_search(erq_plan* p, const float* queries, uint64_t nq, uint32_t* ids,
                           float* dists, uint32_t* nprobe_used, void* stream) {
    if (!p) return fail(ERQ_ERR_INVALID_ARGUMENT, "plan is NULL");
    if (nq == 0) return ERQ_OK;
    if (!queries || !ids) return fail(ERQ_ERR_INVALID_ARGUMENT, "queries and ids are required");
    if (nq > p->max_batch)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "batch of %llu exceeds the plan's max_batch %llu",
                    (unsigned long long)nq, (unsigned long long)p->max_batch);
    std::lock_guard<std::mutex> g(p->mu);
    DeviceGuard guard;
    ERQ_TRY(guard.set(p->idx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool host = !is_device_ptr(ids) || (dists && !is_device_ptr(dists)) ||
                      (nprobe_used && !is_device_ptr(nprobe_used)) || !is_device_ptr(queries);
    const uint64_t chunks = host ? plan_chunks(p, nq) : 1;
    for (int sl = 0; sl < 2; ++sl)  // a synchronous call orders after any earlier async one
        if (p->slot_used[sl]) ERQ_CUDA(cudaStreamWaitEvent(st, p->ev_comp[sl], 0));
    if (chunks > 1) {
        ERQ_TRY(plan_search_pipelined(p, queries, nq, chunks, ids, dists, nprobe_used, st));
    } else {
        if (p->use_graphs) {  // capture (first use) before staging: capture runs nothing
            cudaGraphExec_t ge = nullptr;
            ERQ_TRY(plan_graph(p, nq, 0, &ge));
        }
        ERQ_TRY(plan_stage_queries(p, queries, nq, st));
        ERQ_TRY(plan_run(p, nq, 0, st));
        ERQ_CUDA(cudaMemcpyAsync(ids, p->ids, nq * p->k * sizeof(uint32_t), cudaMemcpyDefault, st));
        if (dists)
            ERQ_CUDA(cudaMemcpyAsync(dists, p->dists, nq * p->k * sizeof(float), cudaMemcpyDefault, st));
        if (nprobe_used)  // a plan without a model keeps nprobe in every entry
            ERQ_CUDA(cudaMemcpyAsync(nprobe_used, p->used, nq * sizeof(uint32_t), cudaMemcpyDefault, st));
    }
    if (host) {
        uint32_t* hw = nullptr;
        ERQ_TRY(tc_status_fetch(st, &hw));
        ERQ_CUDA(cudaStreamSynchronize(st));
        ERQ_TRY(tc_status_check(hw));
    }
    return ERQ_OK;
}

uint64_t erq_plan_device_bytes(const erq_plan* p) { return p ? p->arena.bytes : 0; }

erq_status erq_plan_search_async(erq_plan* p, const float* queries, uint64_t nq, uint32_t* ids,
                                 float* dists, uint32_t* nprobe_used, void* stream) {
    if (!p) return fail(ERQ_ERR_INVALID_ARGUMENT, "plan is NULL");
    if (nq == 0) return ERQ_OK;
    if (!queries || !ids) return fail(ERQ_ERR_INVALID_ARGUMENT, "queries and ids are required");
    if (nq > p->max_batch)
        return fail(ERQ_ERR_INVALID_ARGUMENT, "batch of %llu exceeds the plan's max_batch %llu",
                    (unsigned long long)nq, (unsigned long long)p->max_batch);
    std::lock_guard<std::mutex> g(p->mu);
    DeviceGuard guard;
    ERQ_TRY(guard.set(p->idx->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int slot = p->next_slot;
    p->next_slot ^= 1;
    const uint64_t cols = p->raw ? p->idx->DIM : p->idx->D;
    // queries in on the copy stream, once the slot's last search has read them
    if (p->slot_used[slot]) ERQ_CUDA(cudaStreamWaitEvent(p->h2d, p->ev_comp[slot], 0));
    ERQ_CUDA(cudaMemcpyAsync(slot ? p->qin1 : p->qin, queries, nq * cols * sizeof(float),
                             cudaMemcpyDefault, p->h2d));
    ERQ_CUDA(cudaEventRecord(p->ev_in[slot], p->h2d));
    // the search and the results out on the caller's stream
    ERQ_CUDA(cudaStreamWaitEvent(st, p->ev_in[slot], 0));
    ERQ_TRY(plan_run(p, nq, slot, st));
    ERQ_CUDA(cudaEventRecord(p->ev_comp[slot], st));
    p->slot_used[slot] = true;
    ERQ_CUDA(cudaMemcpyAsync(ids, slot ? p->ids1 : p->ids, nq * p->k * sizeof(uint32_t),
                             cudaMemcpyDefault, st));
    if (dists)
        ERQ_CUDA(cudaMemcpyAsync(dists, slot ? p->dists1 : p->dists, nq * p->k * sizeof(float),
                                 cudaMemcpyDefault, st));
    if (nprobe_used)
        ERQ_CUDA(cudaMemcpyAsync(nprobe_used, slot ? p->used1 : p->used, nq * sizeof(uint32_t),
                                 cudaMemcpyDefault, st));
    return ERQ_OK;
}

erq_status erq_plan_set_pipeline(erq_plan* p, int chunks) {
    if (!p) return fail(ERQ_ERR_INVALID_ARGUMENT, "plan is NULL");
    if (chunks < 0 || chunks > 64) return fail(ERQ_ERR_INVALID_ARGUMENT, "chunks outside 0..64");
    std::lock_guard<std::mutex> g(p->mu);
    p->pipe_chunks = chunks;
    return ERQ_OK;
}

erq_status erq_plan_set_graphs(erq_plan* p, int on) {
    if (!p) return fail(ERQ_ERR_INVALID_ARGUMENT, "plan is NULL");
    std::lock_guard<std::mutex> g(p->mu);
    p->use_graphs = on != 0;
    return ERQ_OK;
}

}  // extern "C"
