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

}  // namespace erq
