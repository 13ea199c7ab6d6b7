// Device helpers for the ME8Q code streams (layout in me8q.h): words of a
// vector's stream, bit fields, and one run's 8-dim block.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace e8qc {

__device__ __forceinline__ uint32_t* me8q_word_ptr(uint4* codes, int nch, size_t slot, int w) {
    return reinterpret_cast<uint32_t*>(codes + ((slot >> 5) * nch + (w >> 2)) * 32 + (slot & 31)) + (w & 3);
}

__device__ __forceinline__ uint32_t me8q_word(const uint4* codes, int nch, size_t slot, int w) {
    return __ldg(reinterpret_cast<const uint32_t*>(codes + ((slot >> 5) * nch + (w >> 2)) * 32 + (slot & 31)) +
                 (w & 3));
}

// Field of `width` (<= 13) bits at bit `pos` of a run starting at word0.
__device__ __forceinline__ uint32_t me8q_bits(const uint4* codes, int nch, size_t slot, int word0, int pos,
                                              int width) {
    const int w = word0 + (pos >> 5), sh = pos & 31;
    uint32_t v = me8q_word(codes, nch, slot, w) >> sh;
    if (sh + width > 32) v |= me8q_word(codes, nch, slot, w + 1) << (32 - sh);
    return v & ((1u << width) - 1u);
}

// Digits and branch of block j of a run at `bits` bits per digit: digit i at
// bits i*b of the block's field, digit 7's lowest bit holding the branch (its
// real lowest bit is the parity of digits 0..6).
__device__ __forceinline__ int me8q_block(const uint4* codes, int nch, size_t slot, int word0, int bits, int j,
                                          uint32_t dg[8]) {
    const int base = j * 8 * bits;
    uint32_t par = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        dg[i] = me8q_bits(codes, nch, slot, word0, base + i * bits, bits);
        par ^= dg[i];
    }
    const uint32_t f7 = me8q_bits(codes, nch, slot, word0, base + 7 * bits, bits);
    dg[7] = (f7 & ~1u) | (par & 1u);
    return static_cast<int>(f7 & 1u);
}

}  // namespace e8qc
