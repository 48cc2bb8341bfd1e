// Index layout in HBM and the kernel that builds it from the file bytes.
//
// File layout of one FastScan block (HIGH_ACC_FAST_SCAN, written by
// DataQuantizer::quantize, inc/index/Quantizer.hpp:276-289, packed by
// pack_codes, inc/index/fastscan/pack_codes.hpp:33-98):
//   bytes [0, 4D):      D/4 groups of 16 bytes; group g = dims 4g..4g+3;
//                        byte j of a group: low nibble = vector perm0[j],
//                        high nibble = vector perm0[j]+16,
//                        perm0 = {0,8,1,9,...,7,15}; nibble bit 3 = dim 4g+0
//   bytes [4D, 4D+128): 32 floats ||o - c|| (one per vector, vector order)
//
// Device layout (chosen for the scan kernel):
//   codes: one 4D-byte block per 32 vectors, regrouped per 64-dim chunk c
//          (groups 16c..16c+15, 256 bytes) so that warp lane L = 16h + j
//          loads 8 contiguous bytes = byte j of groups 16c+8h+0..7:
//            dev[c*256 + L*8 + u] = file[(16c + 8h + u)*16 + j]
//          A warp reads one chunk with one coalesced 256-byte load, every
//          half-warp then walks one group at a time (16 lanes sharing one
//          16-entry table: broadcast-friendly shared-memory lookups).
//   onorm: 32 floats per block, split out of the block.
//
// EX-bit codes.  File layout: one row of D*EX/8 bytes per vector, 64-dim
// groups of 8*EX bytes (store_compacted_code, inc/index/Quantizer.hpp:491-631).
// Device layout (chosen for the refinement kernel, where the 4 lanes r = 0..3
// of a quad compute one candidate's inner product): lane r owns the dims
// 16s + 4r + i (i = 0..3, steps s = 0..D/16-1), which are the dims of the
// reference's accumulators 4r..4r+3.  Codes are stored in SB = 8 (EX >= 5),
// 4 (EX = 3, 4) or 2 (EX = 2) bits; lane r's stream of 32-bit words holds
//   SB = 8: word s, byte i = code of dim 16s + 4r + i
//   SB = 4: word j, byte i: low nibble = step 2j, high nibble = step 2j + 1
//   SB = 2: word j, byte i: bits 2t..2t+1 = step 4j + t
// padded with zeros to U whole uint4s; uint4 u of lane r sits at byte
// 16 * (4u + r) of the row, so a quad reads 64 contiguous bytes per load.
// Rows are 64 * U bytes.
#pragma once

#include "common.cuh"

namespace erq {

// One thread per output byte of the code region.
__global__ void transform_blocks_kernel(const uint8_t* __restrict__ raw,
                                        uint8_t* __restrict__ codes,
                                        float* __restrict__ onorm, uint64_t nblocks, int D) {
    const uint64_t code_bytes = 4ull * D;
    const uint64_t raw_block = code_bytes + kFastSize * sizeof(float);
    const uint64_t total = nblocks * code_bytes;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = i / code_bytes;
        const uint32_t r = (uint32_t)(i - b * code_bytes);
        const uint32_t c = r >> 8;          // 64-dim chunk
        const uint32_t L = (r >> 3) & 31;   // lane
        const uint32_t u = r & 7;           // byte within the lane's 8
        const uint32_t h = L >> 4, j = L & 15;
        const uint32_t g = 16 * c + 8 * h + u;
        codes[i] = raw[b * raw_block + 16ull * g + j];
    }
    const uint64_t nf = nblocks * kFastSize;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nf;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = i / kFastSize;
        const uint32_t v = (uint32_t)(i - b * kFastSize);
        float f;
        memcpy(&f, raw + b * raw_block + code_bytes + 4ull * v, sizeof(float));
        onorm[i] = f;
    }
}

// Storage bits per code and row bytes of the device EX-code layout.
__host__ __device__ constexpr int ex_storage_bits(int EX) { return EX >= 5 ? 8 : (EX >= 3 ? 4 : 2); }
__host__ __device__ constexpr int ex_steps_per_uint4(int EX) { return 32 / ex_storage_bits(EX); }
__host__ __device__ constexpr uint64_t ex_row_uint4(int D, int EX) {
    return ((uint64_t)(D / 16) + ex_steps_per_uint4(EX) - 1) / ex_steps_per_uint4(EX);
}
__host__ __device__ constexpr uint64_t ex_row_bytes(int D, int EX) { return 64 * ex_row_uint4(D, EX); }

// Four consecutive dims (16*sub + 4*qd .. +3 of a 64-dim group) of one EX-bit
// code as bytes of a word.  `w` holds the group's 8*EX bytes as 2*EX words.
// Layouts: store_compacted_code, inc/index/Quantizer.hpp:491-631.
template <int EX>
__device__ __forceinline__ uint32_t ex_quad(const uint32_t* w, int sub, int qd) {
    if (EX == 8) {
        return w[4 * sub + qd];
    } else if (EX == 4) {  // per 32 dims: 16 bytes, low nibble = dims 0-15
        const uint32_t c = w[4 * (sub >> 1) + qd];
        return (sub & 1) ? ((c >> 4) & 0x0F0F0F0Fu) : (c & 0x0F0F0F0Fu);
    } else if (EX == 2 || EX == 3) {  // 2 bits at 2*sub of bytes 0-15
        uint32_t v = (w[qd] >> (2 * sub)) & 0x03030303u;
        if (EX == 3) {
            // bit j of byte m of the top word = bit 2 of dim 8j + m; these
            // dims have m = (4qd .. 4qd+3) % 8 and j = 2*sub + qd/2
            const uint32_t t = w[4 + (qd & 1)];
            const int j = 2 * sub + (qd >> 1);
            v |= ((j <= 2) ? (t << (2 - j)) : (t >> (j - 2))) & 0x04040404u;
        }
        return v;
    } else {  // EX == 6 || EX == 7: c1 = bytes 0-15, c2 = 16-31, c3 = 32-47
        const uint32_t c1 = w[qd], c2 = w[4 + qd], c3 = w[8 + qd];
        uint32_t v;
        if (sub == 0) {
            v = c1 & 0x3F3F3F3Fu;
        } else if (sub == 1) {
            v = c2 & 0x3F3F3F3Fu;
        } else if (sub == 2) {
            v = ((c1 >> 2) & 0x30303030u) | (c3 & 0x0F0F0F0Fu);
        } else {
            v = ((c2 >> 2) & 0x30303030u) | ((c3 >> 4) & 0x0F0F0F0Fu);
        }
        if (EX == 7) {  // bit 6 from the top word (after 48 bytes)
            const uint32_t t = w[12 + (qd & 1)];
            const int j = 2 * sub + (qd >> 1);
            v |= ((j <= 6) ? (t << (6 - j)) : (t >> (j - 6))) & 0x40404040u;
        }
        return v;
    }
}


// File rows -> device rows, one thread per output word (vector, lane, word).
template <int EX>
__global__ void transform_excode_kernel(const uint8_t* __restrict__ file, uint32_t* __restrict__ dev,
                                        uint64_t N, int D) {
    constexpr int SB = ex_storage_bits(EX);
    constexpr int SPW = 8 / SB;  // steps per word
    const uint64_t file_row = (uint64_t)D * EX / 8;
    const uint64_t U = ex_row_uint4(D, EX);
    const uint64_t words_per_row = 16 * U;
    const int steps = D / 16;
    const uint64_t total = N * words_per_row;
    for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < total;
         o += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = o / words_per_row;
        const uint32_t w_in_row = (uint32_t)(o - v * words_per_row);
        const uint32_t u = w_in_row >> 4, r = (w_in_row >> 2) & 3, m = w_in_row & 3;
        const uint32_t j = 4 * u + m;  // word index in lane r's stream
        uint32_t out = 0;
        for (int t = 0; t < SPW; ++t) {
            const int s = (int)j * SPW + t;
            if (s >= steps) break;
            const int g = s >> 2, sub = s & 3;
            uint32_t w[2 * EX];
            const uint8_t* src = file + v * file_row + (uint64_t)g * 8 * EX;
            for (int i = 0; i < 2 * EX; ++i) memcpy(&w[i], src + 4 * i, 4);
            const uint32_t codes = ex_quad<EX>(w, sub, (int)r);  // bytes = dims 16s+4r+i
            out |= codes << (SB * t);
        }
        dev[o] = out;
    }
}

}  // namespace erq
