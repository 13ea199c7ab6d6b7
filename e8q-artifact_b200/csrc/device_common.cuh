// Device helpers shared by the kernels: warp top-k, the FHT-Kac-4 rotation in
// shared memory, and the lattice-code block decode.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace e8qc {

constexpr unsigned kFull = 0xFFFFFFFFu;

// Total order of results: smaller distance first, ties by smaller id
// (src/index/e8q_internal.hpp:47-49).
// (Short-circuit form: measured 0.12 ms faster per 4,096-query precision
// select than the branch-free form, which evaluates the id compare always.)
__device__ __forceinline__ bool better(float d1, uint32_t i1, float d2, uint32_t i2) {
    return d1 < d2 || (d1 == d2 && i1 < i2);
}

// ---------------------------------------------------------------------------
// Warp-wide sorted top-k (k <= 128). Entry j (ascending by `better`) lives in
// lane j % 32, slot j / 32. Offers are filtered against the current k-th
// entry, and each accepted candidate is inserted with one ballot per slot and
// a one-position shift of the tail. All members must be called by the whole
// warp with warp-uniform arguments unless stated.
struct WarpTopK {
    float d[4];
    uint32_t id[4];
    int k;
    float thr_d;
    uint32_t thr_id;

    __device__ void init(int k_) {
        k = k_;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            d[s] = __int_as_float(0x7f800000);
            id[s] = 0xFFFFFFFFu;
        }
        thr_d = __int_as_float(0x7f800000);
        thr_id = 0xFFFFFFFFu;
    }

    __device__ __forceinline__ void refresh_threshold() {
        const int j = k - 1;
        const int s = j >> 5;
        float v = d[0];
        uint32_t w = id[0];
        if (s == 1) { v = d[1]; w = id[1]; }
        if (s == 2) { v = d[2]; w = id[2]; }
        if (s == 3) { v = d[3]; w = id[3]; }
        thr_d = __shfl_sync(kFull, v, j & 31);
        thr_id = __shfl_sync(kFull, w, j & 31);
    }

    // Insert one warp-uniform candidate already known to beat the threshold.
    __device__ void insert(float cd, uint32_t cid) {
        const int lane = threadIdx.x & 31;
        int pos = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) pos += __popc(__ballot_sync(kFull, better(d[s], id[s], cd, cid)));
#pragma unroll
        for (int s = 3; s >= 0; --s) {
            float pd = __shfl_up_sync(kFull, d[s], 1);
            uint32_t pi = __shfl_up_sync(kFull, id[s], 1);
            if (s > 0) {
                const float cd2 = __shfl_sync(kFull, d[s > 0 ? s - 1 : 0], 31);
                const uint32_t ci2 = __shfl_sync(kFull, id[s > 0 ? s - 1 : 0], 31);
                if (lane == 0) { pd = cd2; pi = ci2; }
            }
            const int j = s * 32 + lane;
            if (j > pos) { d[s] = pd; id[s] = pi; }
            else if (j == pos) { d[s] = cd; id[s] = cid; }
        }
        refresh_threshold();
    }

    // Per-lane offer: lane candidate (dist, id) with `want` true where the lane
    // has a candidate. The id is only needed when the distance can tie or beat
    // the threshold, so it is fetched through `get_id` lazily. When several
    // lanes pass and k <= 32, the 32 candidates are bitonic-sorted and merged
    // into the list in one pass; otherwise they are inserted one at a time.
    template <class GetId>
    __device__ void offer(float dist, bool want, GetId get_id) {
        bool maybe = want && !(dist > thr_d);
        uint32_t cid = 0xFFFFFFFFu;
        if (maybe) cid = get_id();
        unsigned m = __ballot_sync(kFull, maybe && better(dist, cid, thr_d, thr_id));
        if (m == 0) return;
        if (k <= 32 && __popc(m) >= 2) {
            const int lane = threadIdx.x & 31;
            const bool in = (m >> lane) & 1u;
            merge32(in ? dist : __int_as_float(0x7f800000), in ? cid : 0xFFFFFFFFu);
            return;
        }
        if (k > 32 && __popc(m) >= 4) {
            const int lane = threadIdx.x & 31;
            const bool in = (m >> lane) & 1u;
            if (k <= 64) merge_wide<2>(in ? dist : __int_as_float(0x7f800000), in ? cid : 0xFFFFFFFFu);
            else merge_wide<4>(in ? dist : __int_as_float(0x7f800000), in ? cid : 0xFFFFFFFFu);
            return;
        }
        while (m) {
            const int src = __ffs(m) - 1;
            const float cd = __shfl_sync(kFull, dist, src);
            const uint32_t ci = __shfl_sync(kFull, cid, src);
            insert(cd, ci);
            m &= ~(1u << src);
            m &= __ballot_sync(kFull, maybe && better(dist, cid, thr_d, thr_id));
        }
    }

    // Bitonic sort of one value per lane across the warp, ascending.
    __device__ __forceinline__ static void sort32(float& cd, uint32_t& ci) {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                const float pd = __shfl_xor_sync(kFull, cd, j);
                const uint32_t pi = __shfl_xor_sync(kFull, ci, j);
                const bool asc = (lane & kk) == 0;
                const bool lower = (lane & j) == 0;
                const bool take = (lower == asc) ? better(pd, pi, cd, ci) : better(cd, ci, pd, pi);
                if (take) {
                    cd = pd;
                    ci = pi;
                }
            }
        }
    }

    // 32 < k <= 32*S: merge one candidate per lane into the S-slot sorted list
    // in one pass. The list (32S ascending) followed by 32S entries that hold
    // the candidates in descending order after 32(S-1) +inf is bitonic; its
    // lower half is min(list, that tail) element-wise -- only the last slot can
    // change -- and a bitonic clean-up of the lower half (slot pairs in
    // registers, then shuffles within each slot) sorts it.
    template <int S>
    __device__ void merge_wide(float cd, uint32_t ci) {
        const int lane = threadIdx.x & 31;
        sort32(cd, ci);
        const float rd = __shfl_sync(kFull, cd, 31 - lane);  // descending
        const uint32_t ri = __shfl_sync(kFull, ci, 31 - lane);
        if (better(rd, ri, d[S - 1], id[S - 1])) {
            d[S - 1] = rd;
            id[S - 1] = ri;
        }
#pragma unroll
        for (int js = S / 2; js >= 1; js >>= 1) {  // distances of 32*js: slot s with slot s + js
#pragma unroll
            for (int s0 = 0; s0 < S; ++s0) {
                if ((s0 & js) == 0) {
                    const int s1 = s0 + js;
                    if (better(d[s1], id[s1], d[s0], id[s0])) {
                        const float td = d[s0];
                        const uint32_t ti = id[s0];
                        d[s0] = d[s1];
                        id[s0] = id[s1];
                        d[s1] = td;
                        id[s1] = ti;
                    }
                }
            }
        }
#pragma unroll
        for (int j = 16; j > 0; j >>= 1) {
            const bool lower = (lane & j) == 0;
#pragma unroll
            for (int s0 = 0; s0 < S; ++s0) {
                const float pd = __shfl_xor_sync(kFull, d[s0], j);
                const uint32_t pi = __shfl_xor_sync(kFull, id[s0], j);
                const bool take = lower ? better(pd, pi, d[s0], id[s0]) : better(d[s0], id[s0], pd, pi);
                if (take) {
                    d[s0] = pd;
                    id[s0] = pi;
                }
            }
        }
        refresh_threshold();
    }

    // k <= 32: merge one candidate per lane into slot 0 (sorted) in one pass:
    // bitonic sort of the candidates, reverse, lane-wise min against the list
    // (the 32 smallest of the union, a bitonic sequence), bitonic clean-up.
    __device__ void merge32(float cd, uint32_t ci) {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                const float pd = __shfl_xor_sync(kFull, cd, j);
                const uint32_t pi = __shfl_xor_sync(kFull, ci, j);
                const bool asc = (lane & kk) == 0;
                const bool lower = (lane & j) == 0;
                const bool take = (lower == asc) ? better(pd, pi, cd, ci) : better(cd, ci, pd, pi);
                if (take) { cd = pd; ci = pi; }
            }
        }
        const float rd = __shfl_sync(kFull, cd, 31 - lane);
        const uint32_t ri = __shfl_sync(kFull, ci, 31 - lane);
        if (better(rd, ri, d[0], id[0])) { d[0] = rd; id[0] = ri; }
#pragma unroll
        for (int j = 16; j > 0; j >>= 1) {
            const float pd = __shfl_xor_sync(kFull, d[0], j);
            const uint32_t pi = __shfl_xor_sync(kFull, id[0], j);
            const bool lower = (lane & j) == 0;
            const bool take = lower ? better(pd, pi, d[0], id[0]) : better(d[0], id[0], pd, pi);
            if (take) { d[0] = pd; id[0] = pi; }
        }
        refresh_threshold();
    }

    __device__ void offer_pair(float dist, uint32_t cid, bool want) {
        offer(dist, want, [&] { return cid; });
    }

    // Entry j of the sorted list (any lane may ask for any j; warp-wide).
    __device__ void store(float* out_d, uint32_t* out_id, int count) const {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int j = s * 32 + lane;
            if (j < count) {
                out_d[j] = d[s];
                out_id[j] = id[s];
            }
        }
    }
};

// ---------------------------------------------------------------------------
// Block-wide bitonic sort (ascending by `better`) of pn entries held in shared
// memory; pn is a power of two, unused entries hold (+inf, UINT32_MAX). All
// threads of the block must call it.
__device__ inline void block_bitonic_sort(float* sd, uint32_t* si, int pn) {
    for (int kk = 2; kk <= pn; kk <<= 1) {
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < pn; i += blockDim.x) {
                const int p = i ^ j;
                if (p > i) {
                    const bool asc = (i & kk) == 0;
                    const float a = sd[i], b = sd[p];
                    const uint32_t ai = si[i], bi = si[p];
                    if (asc ? better(b, bi, a, ai) : better(a, ai, b, bi)) {
                        sd[i] = b;
                        sd[p] = a;
                        si[i] = bi;
                        si[p] = ai;
                    }
                }
            }
            __syncthreads();
        }
    }
}

__host__ __device__ inline int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// ---------------------------------------------------------------------------
// FHT-Kac-4 rotation of `rows` vectors held in shared memory (row stride
// `ld` floats, padded_dim `pd` floats each, already zero-padded past dim).
// Same per-element operations as src/utils/rotator.cpp:53-80 with the
// primitives of src/simd/kernels_generic.cpp:49-77 (sign flip, radix-2
// butterflies stage by stage, x fac, Kac walk (x+y, x-y) over halves, final
// x0.25 when the window is narrower than pd), so the result is bit-exact.
// Every operation is an explicitly rounded intrinsic, so no compiler
// contraction can change a bit. All threads of the block must call it.
__device__ inline void rotate_rows_smem(float* x, int rows, int ld, int pd, int td, float fac,
                                        const uint8_t* __restrict__ signs) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per_round = pd / 8;
    const bool padded = td != pd;
    for (int r = 0; r < 4; ++r) {
        const uint8_t* sg = signs + r * per_round;
        for (int e = tid; e < rows * pd; e += nt) {
            const int row = e / pd, i = e - row * pd;
            if ((sg[i >> 3] >> (i & 7)) & 1) x[row * ld + i] = -x[row * ld + i];
        }
        __syncthreads();
        const int w0 = (!padded || (r & 1) == 0) ? 0 : pd - td;
        const int half = td >> 1;
        for (int h = 1; h < td; h <<= 1) {
            for (int e = tid; e < rows * half; e += nt) {
                const int row = e / half, p = e - row * half;
                const int i = (p / h) * (h << 1) + (p % h);
                float* b = x + row * ld + w0;
                const float a0 = b[i], a1 = b[i + h];
                b[i] = __fadd_rn(a0, a1);
                b[i + h] = __fsub_rn(a0, a1);
            }
            __syncthreads();
        }
        for (int e = tid; e < rows * td; e += nt) {
            const int row = e / td, i = e - row * td;
            x[row * ld + w0 + i] = __fmul_rn(x[row * ld + w0 + i], fac);
        }
        __syncthreads();
        if (padded) {
            const int hp = pd >> 1;
            for (int e = tid; e < rows * hp; e += nt) {
                const int row = e / hp, i = e - row * hp;
                float* b = x + row * ld;
                const float a0 = b[i], a1 = b[i + hp];
                b[i] = __fadd_rn(a0, a1);
                b[i + hp] = __fsub_rn(a0, a1);
            }
            __syncthreads();
        }
    }
    if (padded) {
        for (int e = tid; e < rows * pd; e += nt) {
            const int row = e / pd, i = e - row * pd;
            x[row * ld + i] = __fmul_rn(x[row * ld + i], 0.25f);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Lattice-code block geometry for a rate: a "group" is the smallest run of
// whole blocks that ends on a 16-byte chunk boundary.
__host__ __device__ constexpr int group_blocks(int bits) {
    return (bits & 1) ? 16 : ((bits & 3) == 2 ? 8 : ((bits & 7) == 4 ? 4 : 2));
}
__host__ __device__ constexpr int group_chunks(int bits) {
    return group_blocks(bits) * 8 * bits / 128;
}

// Field of W bits at bit offset `off` of a little-endian word array (one
// spare word past the end). Offsets are compile-time after unrolling.
__device__ __forceinline__ uint32_t field(const uint32_t* w, int off, int width) {
    const uint32_t v = __funnelshift_r(w[off >> 5], w[(off >> 5) + 1], off & 31);
    return width >= 32 ? v : (v & ((1u << width) - 1u));
}

// Decode block `blk` (bit offset blk*8*BITS in w) into digits and branch:
// digit i is the field at i*BITS, digit 7's LSB slot is the branch and its
// real LSB is the parity of digits 0..6.
template <int BITS>
__device__ __forceinline__ int decode_block(const uint32_t* w, int base, uint32_t dig[8]) {
    uint32_t par = 0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        dig[i] = field(w, base + i * BITS, BITS);
        par ^= dig[i];
    }
    const uint32_t f7 = field(w, base + 7 * BITS, BITS);
    dig[7] = (f7 & ~1u) | (par & 1u);
    return static_cast<int>(f7 & 1u);
}

}  // namespace e8qc
