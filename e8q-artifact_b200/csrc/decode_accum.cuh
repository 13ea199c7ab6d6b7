// Decode + accumulate of packed E8Q blocks against an fp32 query, shared by
// the plain scan and the precision path's exact rescoring.
//
// A lane decodes one vector: 8 digits per block, digit 7's stored LSB is the
// branch and its real LSB the parity of digits 0..6; level values are gathered
// from a shared-memory table replicated table_rep(bits) times (entry e of
// copy c at byte (e * REP + c) * 4), and each block contributes 8 FMAs into
// one of two alternating accumulators (even blocks acc0, odd blocks acc1).
#pragma once

#include <stdint.h>

#include "device_common.cuh"
#include "scan_plain.h"

namespace e8qc {

__device__ __forceinline__ float lds_f32(uint32_t addr) {
    float v;
    asm("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
    return v;
}

// log2 of the byte stride between consecutive level entries: REP per-lane
// copies of 4 bytes each.
__host__ __device__ constexpr int entry_shift(int bits) {
    return table_rep(bits) == 32 ? 7 : table_rep(bits) == 16 ? 6 : table_rep(bits) == 8 ? 5
         : table_rep(bits) == 4 ? 4 : table_rep(bits) == 2 ? 3 : 2;
}

// Field of WIDTH bits at bit offset OFF of w[], returned already shifted to a
// byte offset into the table (left by SH = entry_shift).
template <int OFF, int WIDTH, int SH>
__device__ __forceinline__ uint32_t field_xs(const uint32_t* w) {
    constexpr int wi = OFF >> 5, sh = OFF & 31;
    constexpr uint32_t m = ((1u << WIDTH) - 1u) << SH;
    if constexpr (sh >= SH) {
        return __funnelshift_r(w[wi], w[wi + 1], sh - SH) & m;
    } else {
        return (w[wi] << (SH - sh)) & m;
    }
}

// One block: 8 digits (digit 7's LSB = parity of digits 0..6, its stored LSB
// slot = branch) -> 8 level gathers from this lane's table copy -> 8 FMAs.
template <int BITS, int OFF>
__device__ __forceinline__ void block_fma(const uint32_t* w, uint32_t tb_addr, const float4 qa, const float4 qb,
                                          float& acc) {
    constexpr int SH = entry_shift(BITS);
    constexpr uint32_t LSB = 1u << SH;
    const uint32_t f0 = field_xs<OFF + 0 * BITS, BITS, SH>(w);
    const uint32_t f1 = field_xs<OFF + 1 * BITS, BITS, SH>(w);
    const uint32_t f2 = field_xs<OFF + 2 * BITS, BITS, SH>(w);
    const uint32_t f3 = field_xs<OFF + 3 * BITS, BITS, SH>(w);
    const uint32_t f4 = field_xs<OFF + 4 * BITS, BITS, SH>(w);
    const uint32_t f5 = field_xs<OFF + 5 * BITS, BITS, SH>(w);
    const uint32_t f6 = field_xs<OFF + 6 * BITS, BITS, SH>(w);
    const uint32_t f7 = field_xs<OFF + 7 * BITS, BITS, SH>(w);
    const uint32_t par = f0 ^ f1 ^ f2 ^ f3 ^ f4 ^ f5 ^ f6;      // bit SH = parity
    const uint32_t d7 = (f7 & ~LSB) | (par & LSB);
    const uint32_t base = tb_addr + ((f7 & LSB) << BITS);        // branch table
    acc = __fmaf_rn(qa.x, lds_f32(base + f0), acc);
    acc = __fmaf_rn(qa.y, lds_f32(base + f1), acc);
    acc = __fmaf_rn(qa.z, lds_f32(base + f2), acc);
    acc = __fmaf_rn(qa.w, lds_f32(base + f3), acc);
    acc = __fmaf_rn(qb.x, lds_f32(base + f4), acc);
    acc = __fmaf_rn(qb.y, lds_f32(base + f5), acc);
    acc = __fmaf_rn(qb.z, lds_f32(base + f6), acc);
    acc = __fmaf_rn(qb.w, lds_f32(base + d7), acc);
}

template <int BITS, int NBLK, int B0>
struct BlockRun {
    __device__ __forceinline__ static void run(const uint32_t* w, uint32_t tb_addr, const float4* sq4, int qblk,
                                               float& acc0, float& acc1) {
        if constexpr (B0 < NBLK) {
            const float4 qa = sq4[2 * (qblk + B0)], qb = sq4[2 * (qblk + B0) + 1];
            block_fma<BITS, B0 * 8 * BITS>(w, tb_addr, qa, qb, (B0 & 1) ? acc1 : acc0);
            BlockRun<BITS, NBLK, B0 + 1>::run(w, tb_addr, sq4, qblk, acc0, acc1);
        }
    }
};

// Decode + accumulate NBLK consecutive blocks whose NCH chunks start at
// `sbuf` (chunk c of the vector at sbuf[c * STRIDE + lane]: STRIDE 32 for
// chunk-row-major tiles, 1 with lane 0 for one vector's contiguous chunks);
// query blocks start at `qblk`.
template <int BITS, int NBLK, int NCH, int STRIDE = 32>
__device__ __forceinline__ void accumulate_blocks(const uint4* __restrict__ sbuf, int lane,
                                                  const float4* __restrict__ sq4, int qblk, uint32_t tb_addr,
                                                  float& acc0, float& acc1) {
    uint32_t w[4 * NCH + 1];
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
        const uint4 v = sbuf[c * STRIDE + lane];
        w[4 * c] = v.x;
        w[4 * c + 1] = v.y;
        w[4 * c + 2] = v.z;
        w[4 * c + 3] = v.w;
    }
    w[4 * NCH] = 0;
    BlockRun<BITS, NBLK, 0>::run(w, tb_addr, sq4, qblk, acc0, acc1);
}

// Decode + accumulate NBLK consecutive blocks from NCH chunks held in
// registers (the same words accumulate_blocks reads from memory).
template <int BITS, int NBLK, int NCH>
__device__ __forceinline__ void accumulate_regs(const uint4 (&v)[NCH], const float4* __restrict__ sq4, int qblk,
                                                uint32_t tb_addr, float& acc0, float& acc1) {
    uint32_t w[4 * NCH + 1];
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
        w[4 * c] = v[c].x;
        w[4 * c + 1] = v[c].y;
        w[4 * c + 2] = v[c].z;
        w[4 * c + 3] = v[c].w;
    }
    w[4 * NCH] = 0;
    BlockRun<BITS, NBLK, 0>::run(w, tb_addr, sq4, qblk, acc0, acc1);
}

}  // namespace e8qc
