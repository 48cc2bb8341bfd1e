/* CPU oracle for the Extended-RaBitQ IVF search path (test infrastructure;
 * see erq_oracle.h).  Compile with -ffp-contract=off, no -ffast-math. */
#include "erq_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define FAST_SIZE 32u

struct orc_index {
    uint64_t N, DIM, D, K, EX;
    uint64_t* sizes;      /* K */
    uint64_t* first_block; /* K */
    uint64_t* first_vec;  /* K */
    float* P;             /* D*D */
    float* centroids;     /* K*D, rotated */
    uint8_t* short_data;  /* total_blocks * block_bytes */
    uint8_t* long_code;   /* N * D*EX/8 */
    float* xipnorm;       /* N */
    uint32_t* ids;        /* N */
    uint64_t total_blocks;
    uint64_t block_bytes; /* 4D + 32*4 (one factor per vector) */
    uint64_t code_len;    /* D*EX/8 */
};

/* ---------------------------------------------------------------- helpers */

/* _mm512_reduce_add_ps as GCC 13 expands it (avx512fintrin.h): halves
 * (l, l+8), then (l, l+4), then (0,2),(1,3), then the final pair. */
static float tree16(const float* a) {
    float t3[8], t6[4];
    for (int l = 0; l < 8; ++l) t3[l] = a[l + 8] + a[l];
    for (int m = 0; m < 4; ++m) t6[m] = t3[m + 4] + t3[m];
    float t80 = t6[0] + t6[2];
    float t81 = t6[1] + t6[3];
    return t80 + t81;
}

/* lowbit / bit_id (inc/defines.hpp:10-11) */
static uint32_t lowbit_u32(uint32_t x) { return x & (0u - x); }

/* ------------------------------------------------------------- index load */

static int read_exact(FILE* f, void* dst, size_t n) { return fread(dst, 1, n, f) == n ? 0 : -1; }

int orc_index_load(const char* path, orc_index** out) {
    *out = NULL;
    FILE* f = fopen(path, "rb");
    if (!f) return -1;
    orc_index* idx = (orc_index*)calloc(1, sizeof(orc_index));
    if (!idx) {
        fclose(f);
        return -6;
    }
    uint64_t hdr[4];
    int rc = 0;
    if (read_exact(f, hdr, sizeof(hdr))) {
        rc = -5;
        goto fail;
    }
    idx->N = hdr[0];
    idx->DIM = hdr[1];
    idx->K = hdr[2];
    idx->EX = hdr[3];
    if (idx->DIM == 0 || idx->K == 0 || idx->DIM > (1u << 16) ||
        !(idx->EX == 2 || idx->EX == 3 || idx->EX == 4 || idx->EX == 6 || idx->EX == 7 ||
          idx->EX == 8)) {
        rc = -2;
        goto fail;
    }
    /* K >= 20000: the reference would probe with HNSW (inc/index/IVF.hpp:157-161);
     * files that carry their centroids in the main file are probed here with
     * the Flat search's semantics, as the GPU library does. */
    idx->D = (idx->DIM + 63) / 64 * 64;
    const uint64_t D = idx->D, K = idx->K, N = idx->N;
    idx->sizes = (uint64_t*)malloc(sizeof(uint64_t) * K);
    idx->first_block = (uint64_t*)malloc(sizeof(uint64_t) * K);
    idx->first_vec = (uint64_t*)malloc(sizeof(uint64_t) * K);
    if (!idx->sizes || !idx->first_block || !idx->first_vec) {
        rc = -6;
        goto fail;
    }
    if (read_exact(f, idx->sizes, sizeof(uint64_t) * K)) {
        rc = -5;
        goto fail;
    }
    uint64_t tot = 0, blocks = 0;
    for (uint64_t c = 0; c < K; ++c) {
        idx->first_block[c] = blocks;
        idx->first_vec[c] = tot;
        tot += idx->sizes[c];
        blocks += (idx->sizes[c] + FAST_SIZE - 1) / FAST_SIZE;
    }
    if (tot != N) {
        rc = -3;
        goto fail;
    }
    idx->total_blocks = blocks;
    idx->block_bytes = 4 * D + FAST_SIZE * sizeof(float);
    idx->code_len = D * idx->EX / 8;
    idx->P = (float*)malloc(sizeof(float) * D * D);
    idx->centroids = (float*)malloc(sizeof(float) * K * D);
    idx->short_data = (uint8_t*)malloc(blocks * idx->block_bytes + 64);
    idx->long_code = (uint8_t*)malloc(N * idx->code_len + 64);
    idx->xipnorm = (float*)malloc(sizeof(float) * N + 64);
    idx->ids = (uint32_t*)malloc(sizeof(uint32_t) * N + 64);
    if (!idx->P || !idx->centroids || !idx->short_data || !idx->long_code || !idx->xipnorm ||
        !idx->ids) {
        rc = -6;
        goto fail;
    }
    if (read_exact(f, idx->P, sizeof(float) * D * D) ||
        read_exact(f, idx->centroids, sizeof(float) * K * D) ||
        read_exact(f, idx->short_data, blocks * idx->block_bytes) ||
        read_exact(f, idx->long_code, N * idx->code_len) ||
        read_exact(f, idx->xipnorm, sizeof(float) * N) ||
        read_exact(f, idx->ids, sizeof(uint32_t) * N)) {
        rc = -5;
        goto fail;
    }
    fclose(f);
    *out = idx;
    return 0;
fail:
    fclose(f);
    orc_index_free(idx);
    return rc;
}

void orc_index_free(orc_index* idx) {
    if (!idx) return;
    free(idx->sizes);
    free(idx->first_block);
    free(idx->first_vec);
    free(idx->P);
    free(idx->centroids);
    free(idx->short_data);
    free(idx->long_code);
    free(idx->xipnorm);
    free(idx->ids);
    free(idx);
}

void orc_index_info(const orc_index* idx, uint64_t* out) {
    out[0] = idx->N;
    out[1] = idx->DIM;
    out[2] = idx->D;
    out[3] = idx->K;
    out[4] = idx->EX;
}

const float* orc_centroids(const orc_index* idx) { return idx->centroids; }
const float* orc_rotation(const orc_index* idx) { return idx->P; }
const uint64_t* orc_cluster_sizes(const orc_index* idx) { return idx->sizes; }
const uint8_t* orc_long_code(const orc_index* idx, uint64_t pos) {
    return idx->long_code + pos * idx->code_len;
}

/* ------------------------------------------------------- coarse quantiser */

/* L2Sqr16 (inc/utils/space.hpp:18-39): lane l accumulates fma(t, t, acc[l])
 * over dims l, l+16, l+32, ... in order; then the reduce tree. */
float orc_l2sqr16(const float* x, const float* y, uint64_t L) {
    float acc[16] = {0};
    for (uint64_t i = 0; i < L; i += 16)
        for (int l = 0; l < 16; ++l) {
            float t = x[i + l] - y[i + l];
            acc[l] = fmaf(t, t, acc[l]);
        }
    return tree16(acc);
}

typedef struct {
    uint32_t id;
    float d;
} cand_t;

static int cand_cmp(const void* a, const void* b) {
    const cand_t* x = (const cand_t*)a;
    const cand_t* y = (const cand_t*)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

/* FlatInitializer::centroids_distances (inc/index/Initializer.hpp:55-68) */
void orc_probe(const orc_index* idx, const float* q, uint64_t nprobe, uint32_t* cids,
               float* sqr_y) {
    const uint64_t K = idx->K, D = idx->D;
    cand_t* all = (cand_t*)malloc(sizeof(cand_t) * K);
    for (uint64_t c = 0; c < K; ++c) {
        all[c].id = (uint32_t)c;
        all[c].d = orc_l2sqr16(q, idx->centroids + c * D, D);
    }
    qsort(all, K, sizeof(cand_t), cand_cmp);
    for (uint64_t i = 0; i < nprobe && i < K; ++i) {
        cids[i] = all[i].id;
        sqr_y[i] = all[i].d;
    }
    free(all);
}

/* ------------------------------------------------- per-(query,cluster) prep */

/* normalize_query16 (inc/utils/space.hpp:749-778),
 * high_acc_quantize16 (inc/utils/space.hpp:695-711),
 * pack_high_acc_LUT (inc/index/HASearcher.hpp:128-185; tables kept as int32
 * without the per-group unsigned shift, which cancels in the sums). */
void orc_prepare(uint64_t D, const float* q, const float* c, float sqr_y, float* unit_q,
                 int16_t* qq, float* delta, float* sumq, int32_t* lut) {
    const float y = sqrtf(sqr_y);
    const float eps = 1e-5f;
    if (y > eps) {
        const float fac = (float)(1.0 / (double)y);
        float acc[16] = {0};
        for (uint64_t i = 0; i < D; i += 16)
            for (int l = 0; l < 16; ++l) {
                float u = (q[i + l] - c[i + l]) * fac;
                unit_q[i + l] = u;
                acc[l] = acc[l] + u;
            }
        *sumq = tree16(acc);
    } else {
        const float v = (float)(1.0 / (double)sqrtf((float)D));
        for (uint64_t i = 0; i < D; ++i) unit_q[i] = v;
        *sumq = (float)D * v;
    }
    /* data_range16: lane-wise max/min seeded with 0, then reduced */
    float vr = 0.0f, vl = 0.0f;
    for (uint64_t i = 0; i < D; ++i) {
        float u = unit_q[i];
        vr = u > vr ? u : vr;
        vl = u < vl ? u : vl;
    }
    const float avl = fabsf(vl), avr = fabsf(vr);
    const float vmax = avl < avr ? avr : avl;
    const float width = vmax / 8191.0f;
    *delta = width;
    for (uint64_t i = 0; i < D; ++i) {
        float t = unit_q[i] / width;
        qq[i] = (int16_t)((double)t + 0.5 - (double)(t < 0));
    }
    /* group g covers dims 4g..4g+3; table index bit 3 selects dim 4g+0,
     * bit 0 selects dim 4g+3 */
    for (uint64_t g = 0; g < D / 4; ++g) {
        int32_t* t = lut + 16 * g;
        const int16_t* x = qq + 4 * g;
        for (int j = 0; j < 16; ++j) {
            int32_t s = 0;
            if (j & 8) s += x[0];
            if (j & 4) s += x[1];
            if (j & 2) s += x[2];
            if (j & 1) s += x[3];
            t[j] = s;
        }
    }
}

/* ------------------------------------------------------------------ scan */

/* Block layout written by pack_codes (inc/index/fastscan/pack_codes.hpp:33-98):
 * group g occupies bytes [16g, 16g+16); byte j holds vector perm0[j] in its
 * low nibble and vector perm0[j]+16 in its high nibble, with
 * perm0 = {0,8,1,9,...,7,15}.  Within a nibble bit 3 is dim 4g+0. */
void orc_block_sums(uint64_t D, const uint8_t* codes, const int32_t* lut, int32_t* S) {
    static const int perm0[16] = {0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15};
    for (int v = 0; v < 32; ++v) S[v] = 0;
    for (uint64_t g = 0; g < D / 4; ++g) {
        const uint8_t* b = codes + 16 * g;
        const int32_t* t = lut + 16 * g;
        for (int j = 0; j < 16; ++j) {
            S[perm0[j]] += t[b[j] & 15];
            S[perm0[j] + 16] += t[b[j] >> 4];
        }
    }
}

typedef struct {
    float c1, c2, c3; /* lower-bound constants */
} lb_consts;

/* constants of accumulate_one_block_high_acc
 * (inc/index/fastscan/FastScan.hpp:295-303); one_over_sqrtD as in
 * inc/index/HASearcher.hpp:56 */
static lb_consts make_lb_consts(uint64_t D, float sumq, float y) {
    const float const_bound = 0.58f;
    const float one_over_sqrtD = (float)(1.0 / (double)sqrtf((float)D));
    lb_consts k;
    k.c1 = (float)(0.5 * (double)sumq - (double)const_bound);
    k.c2 = ((float)-5 * y) * one_over_sqrtD;
    k.c3 = y * y;
    return k;
}

/* lower bound of one lane (inc/index/fastscan/FastScan.hpp:309-323) */
static float lane_lb(float ipq, float onorm, lb_consts k) {
    float t = ipq - k.c1;
    t = t * k.c2;
    t = t * onorm;
    t = t + k.c3;
    t = t + onorm * onorm;
    return t;
}

uint64_t orc_scan_cluster(const orc_index* idx, const float* q, uint32_t cid, float sqr_y,
                          float distk, int32_t* S, float* ipq, uint32_t* masks) {
    const uint64_t D = idx->D;
    float* unit_q = (float*)malloc(sizeof(float) * D);
    int16_t* qq = (int16_t*)malloc(sizeof(int16_t) * D);
    int32_t* lut = (int32_t*)malloc(sizeof(int32_t) * 4 * D);
    float delta, sumq;
    const float y = sqrtf(sqr_y);
    orc_prepare(D, q, idx->centroids + (uint64_t)cid * D, sqr_y, unit_q, qq, &delta, &sumq, lut);
    const lb_consts k = make_lb_consts(D, sumq, y);
    const uint64_t nb = (idx->sizes[cid] + FAST_SIZE - 1) / FAST_SIZE;
    for (uint64_t b = 0; b < nb; ++b) {
        const uint8_t* blk = idx->short_data + (idx->first_block[cid] + b) * idx->block_bytes;
        const float* onorm = (const float*)(blk + 4 * D);
        int32_t s[32];
        orc_block_sums(D, blk, lut, s);
        uint32_t m = 0;
        for (int v = 0; v < 32; ++v) {
            float ip = (float)s[v] * delta;
            S[32 * b + v] = s[v];
            ipq[32 * b + v] = ip;
            if (lane_lb(ip, onorm[v], k) < distk) m |= 1u << v;
        }
        masks[b] = m;
    }
    free(unit_q);
    free(qq);
    free(lut);
    return nb;
}

/* ------------------------------------------------------------ EX codes */

/* bit (8m + j) of an 8-byte top-bit word holds dim 8j + m of the 64 dims
 * (store_compacted_code, inc/index/Quantizer.hpp:579-585,619-625) */
static int top_bit(const uint8_t* w8, int d) {
    uint64_t w;
    memcpy(&w, w8, 8);
    return (int)((w >> (8 * (d % 8) + d / 8)) & 1u);
}

void orc_ex_decode(uint64_t D, uint64_t EX, const uint8_t* code, uint8_t* out) {
    switch (EX) {
        case 8:
            memcpy(out, code, D);
            break;
        case 4: /* per 32 dims: 16 bytes, dims 0-15 low nibbles, 16-31 high */
            for (uint64_t i = 0; i < D; i += 32, code += 16)
                for (int l = 0; l < 16; ++l) {
                    out[i + l] = code[l] & 15;
                    out[i + 16 + l] = code[l] >> 4;
                }
            break;
        case 2: /* per 64 dims: 16 bytes, dim 16s+l at bits 2s..2s+1 of byte l */
        case 3: /* EX2 layout of the low 2 bits, then 8 bytes of bit 2 */
            for (uint64_t i = 0; i < D; i += 64) {
                for (int l = 0; l < 16; ++l)
                    for (int s = 0; s < 4; ++s) out[i + 16 * s + l] = (code[l] >> (2 * s)) & 3;
                code += 16;
                if (EX == 3) {
                    for (int d = 0; d < 64; ++d) out[i + d] |= (uint8_t)(top_bit(code, d) << 2);
                    code += 8;
                }
            }
            break;
        case 6: /* per 64 dims: 48 bytes */
        case 7: /* EX6 layout of the low 6 bits, then 8 bytes of bit 6 */
            for (uint64_t i = 0; i < D; i += 64) {
                const uint8_t* c1 = code;
                const uint8_t* c2 = code + 16;
                const uint8_t* c3 = code + 32;
                for (int l = 0; l < 16; ++l) {
                    out[i + l] = c1[l] & 63;
                    out[i + 16 + l] = c2[l] & 63;
                    out[i + 32 + l] = (uint8_t)(((c1[l] >> 6) << 4) | (c3[l] & 15));
                    out[i + 48 + l] = (uint8_t)(((c2[l] >> 6) << 4) | (c3[l] >> 4));
                }
                code += 48;
                if (EX == 7) {
                    for (int d = 0; d < 64; ++d) out[i + d] |= (uint8_t)(top_bit(code, d) << 6);
                    code += 8;
                }
            }
            break;
        default:
            memset(out, 0, D);
    }
}

/* IP16_fxu8 / IP32_fxu4 / IP64_fxu{2,3,6,7} (inc/utils/space.hpp:109-131,
 * 152-173, 247-497): every variant feeds dims 16s..16s+15 to lanes 0..15 in
 * ascending s with a fused multiply-add, then the reduce tree. */
float orc_ex_ip(uint64_t D, uint64_t EX, const float* unit_q, const uint8_t* code) {
    uint8_t* v = (uint8_t*)malloc(D);
    orc_ex_decode(D, EX, code, v);
    float acc[16] = {0};
    for (uint64_t i = 0; i < D; i += 16)
        for (int l = 0; l < 16; ++l) acc[l] = fmaf(unit_q[i + l], (float)v[i + l], acc[l]);
    free(v);
    return tree16(acc);
}

/* ---------------------------------------------------------------- top-k */

/* ResultPool (inc/index/Pool.hpp:10-50) */
typedef struct {
    uint32_t* ids;
    float* d;
    uint64_t size, cap;
} pool_t;

/* find_bsearch (inc/index/Pool.hpp:40-49), same probe sequence */
static uint64_t pool_bsearch(const pool_t* p, float dist) {
    uint64_t lo = 0, len = p->size, half;
    while (len > 1) {
        half = len >> 1;
        len -= half;
        lo += (uint64_t)(p->d[lo + half - 1] < dist) * half;
    }
    return (lo < p->size && p->d[lo] < dist) ? lo + 1 : lo;
}

static void pool_insert(pool_t* p, uint32_t u, float dist) {
    if (p->size == p->cap && dist > p->d[p->size - 1]) return;
    uint64_t lo = pool_bsearch(p, dist);
    memmove(&p->ids[lo + 1], &p->ids[lo], (p->size - lo) * sizeof(uint32_t));
    p->ids[lo] = u;
    memmove(&p->d[lo + 1], &p->d[lo], (p->size - lo) * sizeof(float));
    p->d[lo] = dist;
    p->size += (p->size < p->cap);
}

static float pool_distk(const pool_t* p) {
    return p->size == p->cap ? p->d[p->size - 1] : FLT_MAX;
}

/* -------------------------------------------------------------- search */

static void search_impl(const orc_index* idx, const float* q, uint64_t k, uint64_t nprobe,
                        uint32_t* ids, float* dists, uint64_t cap, uint32_t* tr_ids,
                        float* tr_d, uint64_t* tr_n) {
    const uint64_t D = idx->D, EX = idx->EX;
    const int fac_rescale = 1 << EX;
    uint32_t* cids = (uint32_t*)malloc(sizeof(uint32_t) * (nprobe + 1));
    float* sqy = (float*)malloc(sizeof(float) * (nprobe + 1));
    float* unit_q = (float*)malloc(sizeof(float) * D);
    int16_t* qq = (int16_t*)malloc(sizeof(int16_t) * D);
    int32_t* lut = (int32_t*)malloc(sizeof(int32_t) * 4 * D);
    pool_t pool;
    pool.ids = (uint32_t*)calloc(k + 1, sizeof(uint32_t));
    pool.d = (float*)calloc(k + 1, sizeof(float));
    pool.size = 0;
    pool.cap = k;
    uint64_t ntr = 0;

    orc_probe(idx, q, nprobe, cids, sqy);
    for (uint64_t p = 0; p < nprobe && k > 0; ++p) {
        const uint32_t cid = cids[p];
        const float sqr_y = sqy[p];
        const float y = sqrtf(sqr_y);
        float delta, sumq;
        orc_prepare(D, q, idx->centroids + (uint64_t)cid * D, sqr_y, unit_q, qq, &delta, &sumq,
                    lut);
        const lb_consts kc = make_lb_consts(D, sumq, y);
        const uint64_t n = idx->sizes[cid];
        const uint64_t nb = (n + FAST_SIZE - 1) / FAST_SIZE;
        float distk = pool_distk(&pool);
        for (uint64_t b = 0; b < nb; ++b) {
            const uint8_t* blk = idx->short_data + (idx->first_block[cid] + b) * idx->block_bytes;
            const float* onorm = (const float*)(blk + 4 * D);
            const uint64_t npts = (b + 1) * FAST_SIZE <= n ? FAST_SIZE : n - b * FAST_SIZE;
            int32_t s[32];
            float ipq[32];
            orc_block_sums(D, blk, lut, s);
            uint32_t mask = 0;
            for (int v = 0; v < 32; ++v) {
                ipq[v] = (float)s[v] * delta;
                if (lane_lb(ipq[v], onorm[v], kc) < distk) mask |= 1u << v;
            }
            if (npts < 32) mask &= (1u << npts) - 1u;
            while (mask) {
                const uint32_t lb = lowbit_u32(mask);
                const int j = __builtin_ctz(lb);
                mask -= lb;
                const uint64_t pos = idx->first_vec[cid] + b * FAST_SIZE + (uint64_t)j;
                const uint32_t id = idx->ids[pos];
                const float sqr_x = onorm[j] * onorm[j];
                const float ip = orc_ex_ip(D, EX, unit_q, idx->long_code + pos * idx->code_len);
                /* inc/index/HASearcher.hpp:229-232: the bracket and the outer
                 * product are double because (FAC_RESCALE - 0.5) is double */
                const float a = (float)fac_rescale * ipq[j] + ip;
                const double br = (double)a - ((double)fac_rescale - 0.5) * (double)sumq;
                const float xy = idx->xipnorm[pos] * y;
                const float ex_dist = (float)((double)(sqr_x + sqr_y) - (double)xy * br);
                if (tr_ids && ntr < cap) {
                    tr_ids[ntr] = id;
                    tr_d[ntr] = ex_dist;
                }
                ++ntr;
                pool_insert(&pool, id, ex_dist);
                distk = pool_distk(&pool);
            }
        }
    }
    if (ids) memcpy(ids, pool.ids, sizeof(uint32_t) * k);
    if (dists)
        for (uint64_t i = 0; i < k; ++i) dists[i] = i < pool.size ? pool.d[i] : INFINITY;
    if (tr_n) *tr_n = ntr;
    free(cids);
    free(sqy);
    free(unit_q);
    free(qq);
    free(lut);
    free(pool.ids);
    free(pool.d);
}

void orc_search(const orc_index* idx, const float* q, uint64_t k, uint64_t nprobe,
                uint32_t* ids, float* dists) {
    search_impl(idx, q, k, nprobe, ids, dists, 0, NULL, NULL, NULL);
}

void orc_search_batch(const orc_index* idx, const float* q, uint64_t nq, uint64_t k,
                      uint64_t nprobe, uint32_t* ids, float* dists, int nthreads) {
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int64_t i = 0; i < (int64_t)nq; ++i)
        search_impl(idx, q + (uint64_t)i * idx->D, k, nprobe, ids + (uint64_t)i * k,
                    dists ? dists + (uint64_t)i * k : NULL, 0, NULL, NULL, NULL);
}

uint64_t orc_trace(const orc_index* idx, const float* q, uint64_t k, uint64_t nprobe,
                   uint64_t cap, uint32_t* cand_ids, float* cand_dist) {
    uint64_t n = 0;
    search_impl(idx, q, k, nprobe, NULL, NULL, cap, cand_ids, cand_dist, &n);
    return n;
}
