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
// Device layout (chosen for the scan kernels, scan.cuh): dims in groups of
// six, idx_t(v) = sum_{j<6} bit(v, 6t + j) << j (0 past D); per 32-vector
// block, chunks of 16 groups, 512 bytes each: lane v's 16 bytes at 16v, byte
// i = 2 * idx_{16k+i}(v) + 128 * (i & 1) (the entry's byte offset in the
// group's 128-byte table, odd groups in the upper half of a 256-byte window).
//   codes: code_block_bytes(D) = 512 * ceil(ceil(D/6)/16) bytes per block
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
#include "scan.cuh"

namespace erq {

// Byte of a file group's 16 bytes that holds vector v's nibble (low nibble
// for v < 16, high for v >= 16): the inverse of perm0 = {0,8,1,9,...,7,15}
// (inc/index/fastscan/pack_codes.hpp:44).
__device__ __forceinline__ uint32_t fastscan_byte_of(uint32_t v) {
    const uint32_t w = v & 15;
    return w < 8 ? 2 * w : 2 * (w - 8) + 1;
}

// One thread per output byte of the code region.  `factors` per vector in
// the file block (1, or 4 without HIGH_ACC_FAST_SCAN: factor 0 goes to onorm,
// 1-3 to f1..f3); `entry_bytes` of the scan's table entries: 2 (code byte
// 2 idx + 128 (i & 1), scan.cuh) or 4 (code byte 4 idx, lowacc.cuh).
__global__ void transform_blocks_kernel(const uint8_t* __restrict__ raw,
                                        uint8_t* __restrict__ codes,
                                        float* __restrict__ onorm, uint64_t nblocks, int D,
                                        int factors, int entry_bytes, float* __restrict__ f1,
                                        float* __restrict__ f2, float* __restrict__ f3) {
    const uint64_t file_code = 4ull * D;
    const uint64_t raw_block = file_code + kFastSize * sizeof(float) * factors;
    const uint32_t bb = code_block_bytes(D);
    const uint64_t total = nblocks * bb;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = i / bb;
        const uint32_t r = (uint32_t)(i - b * bb);
        const uint32_t k = r >> 9, v = (r >> 4) & 31, byte = r & 15;
        const uint32_t t = 16 * k + byte;
        const uint8_t* fb = raw + b * raw_block;
        const uint32_t jv = fastscan_byte_of(v), hi = v >> 4;
        uint32_t idx = 0;
        for (int j = 0; j < kHexDims; ++j) {
            const uint32_t dim = kHexDims * t + j;
            if (dim >= (uint32_t)D) break;
            const uint32_t g = dim >> 2, rr = dim & 3;
            const uint32_t x = fb[16 * g + jv];
            const uint32_t nib = hi ? (x >> 4) : (x & 15u);
            idx |= ((nib >> (3 - rr)) & 1u) << j;  // nibble bit 3 = dim 4g + 0
        }
        codes[i] = (uint8_t)(entry_bytes == 4 ? 4 * idx : 2 * idx + 128 * (byte & 1));
    }
    const uint64_t nf = nblocks * kFastSize;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nf;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = i / kFastSize;
        const uint32_t v = (uint32_t)(i - b * kFastSize);
        const uint8_t* fac = raw + b * raw_block + file_code;
        float f;
        memcpy(&f, fac + 4ull * v, sizeof(float));
        onorm[i] = f;
        if (factors == 4) {
            memcpy(&f, fac + 4ull * (kFastSize + v), sizeof(float));
            f1[i] = f;
            memcpy(&f, fac + 4ull * (2 * kFastSize + v), sizeof(float));
            f2[i] = f;
            memcpy(&f, fac + 4ull * (3 * kFastSize + v), sizeof(float));
            f3[i] = f;
        }
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
