// Device helpers shared by the one-query scans (plain and pruned): streaming
// loads, the per-rate step geometry of the register-ring decode, probe lookup
// by tile, and the block-wide top-k reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "decode_accum.cuh"
#include "device_common.cuh"
#include "internal.h"
#include "scan_plain.h"
#include "tma.cuh"

namespace e8qc {
namespace scan1 {

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

constexpr int kWarps = 16;      // warps per CTA; one CTA per SM
constexpr int kToffCap = 1024;  // tile offsets cached in shared memory
constexpr int kSelCap = 256;    // survivors ranked by counting

// Streaming 16-byte load: read-only, no L1 allocation (each byte is used once
// per query).
__device__ __forceinline__ uint4 ld_stream(const uint4* p) {
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p));
    return v;
}

template <int NCH>
__device__ __forceinline__ void load_chunks(uint4 (&v)[NCH], const uint4* src) {
#pragma unroll
    for (int c = 0; c < NCH; ++c) v[c] = ld_stream(src + c * 32);
}

// Step geometry of a rate: SBLK blocks in SCH chunks per step; odd rates whose
// block count leaves half a step end with a tail of 8 blocks in TCH chunks.
template <int BITS>
struct StepGeo {
    static constexpr int SBLK = (BITS & 1) ? 16 : 8;
    static constexpr int SCH = SBLK * BITS / 16;
    static constexpr int TCH = (64 * BITS + 127) / 128;
    // register ring depth: about 12-16 chunks in flight per lane (the wide
    // odd rates, 9 bits and up, load each step just before decoding it)
    static constexpr int R = SCH <= 3 ? 4 : (SCH <= 4 ? 3 : (SCH <= 7 ? 2 : 1));
};

// Decode + accumulate steps [s_lo, s_hi) of one vector (and the tail when
// `tail`), streaming the chunks through a register ring of R steps.
// `src` points at chunk 0 of this lane's vector (chunk c at src[c * 32]).
template <int BITS>
__device__ __forceinline__ void scan_steps(const uint4* __restrict__ src, int s_lo, int s_hi, bool tail, int nsteps,
                                           const float4* __restrict__ sq4, uint32_t tb_addr, float& acc0,
                                           float& acc1) {
    using G = StepGeo<BITS>;
    constexpr int R = G::R, SCH = G::SCH, SBLK = G::SBLK, TCH = G::TCH;
    uint4 buf[R][SCH];
    const int n = s_hi - s_lo;
    const uint4* base = src + static_cast<size_t>(s_lo) * SCH * 32;
#pragma unroll
    for (int r = 0; r < R - 1; ++r)
        if (r < n) load_chunks(buf[r], base + r * SCH * 32);
    uint4 tb[(BITS & 1) ? TCH : 1];
    if constexpr ((BITS & 1) != 0) {
        if (tail) load_chunks(tb, src + static_cast<size_t>(nsteps) * SCH * 32);
    }
    for (int i0 = 0; i0 < n; i0 += R) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = i0 + r;
            if (i < n) {
                if (i + R - 1 < n) load_chunks(buf[(r + R - 1) % R], base + (i + R - 1) * SCH * 32);
                accumulate_regs<BITS, SBLK, SCH>(buf[r], sq4, (s_lo + i) * SBLK, tb_addr, acc0, acc1);
            }
        }
    }
    if constexpr ((BITS & 1) != 0) {
        if (tail) accumulate_regs<BITS, 8, TCH>(tb, sq4, nsteps * SBLK, tb_addr, acc0, acc1);
    }
}

// Largest p in [0, nprobe) with off[p] <= t (empty lists share offsets; the
// largest such p is the list that holds tile t).
__device__ __forceinline__ int find_probe(const uint32_t* off, int nprobe, uint32_t t) {
    int lo = 0, hi = nprobe;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The sharper of two upper bounds of the k-th best entry of `nlists`
// sorted lists of k entries each (list L at [L*k, L*k+k)): the best of the
// lists' k-th entries (that list holds k entries at or below it) and, with
// at least k lists, the k-th best of the lists' first entries (k lists each
// hold one). Block-wide (all threads call; the result is in every thread).
__device__ inline void lists_threshold(const float* ld, const uint32_t* lid, int nlists, int k, float& td_out,
                                       uint32_t& ti_out) {
    __shared__ float s_td, s_t2d;
    __shared__ uint32_t s_ti, s_t2i;
    const int tid = threadIdx.x, lane = tid & 31, nt = blockDim.x;
    const int warp = tid >> 5, nw = nt >> 5;
    if (tid == 0) {
        s_t2d = inf_f();
        s_t2i = 0xFFFFFFFFu;
    }
    __syncthreads();
    // warp 0: the best of the lists' k-th entries
    if (warp == 0) {
        float td = inf_f();
        uint32_t ti = 0xFFFFFFFFu;
        for (int L = lane; L < nlists; L += 32) {
            const float d = ld[L * k + k - 1];
            const uint32_t i = lid[L * k + k - 1];
            if (better(d, i, td, ti)) { td = d; ti = i; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float d = __shfl_xor_sync(kFull, td, o);
            const uint32_t i = __shfl_xor_sync(kFull, ti, o);
            if (better(d, i, td, ti)) { td = d; ti = i; }
        }
        if (lane == 0) {
            s_td = td;
            s_ti = ti;
        }
    }
    // the other warps (all, with one warp): the head whose rank among the
    // heads is k - 1 (real heads are unique; padding heads only matter when
    // fewer than k are real). Each warp holds all heads in registers (lane l:
    // heads l, l + 32, ...) and ranks four of its share per step, each with a
    // warp reduction of the lanes' counts.
    constexpr int kHpl = 8;  // heads per lane: up to 256 lists
    const int w0 = nw > 1 ? 1 : 0, nr = nw - w0;
    if (nlists >= k && warp >= w0) {
        if (nlists <= 32 * kHpl) {
            float hd[kHpl];
            uint32_t hi[kHpl];
#pragma unroll
            for (int m = 0; m < kHpl; ++m) {
                const int L = lane + 32 * m;
                hd[m] = L < nlists ? ld[L * k] : inf_f();
                hi[m] = L < nlists ? lid[L * k] : 0xFFFFFFFFu;
            }
            for (int L0 = warp - w0; L0 < nlists; L0 += 4 * nr) {
                int c[4] = {0, 0, 0, 0};
                float d[4];
                uint32_t i[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int L = L0 + u * nr;
                    d[u] = L < nlists ? ld[L * k] : inf_f();
                    i[u] = L < nlists ? lid[L * k] : 0xFFFFFFFFu;
                }
#pragma unroll
                for (int m = 0; m < kHpl; ++m)
#pragma unroll
                    for (int u = 0; u < 4; ++u) c[u] += better(hd[m], hi[m], d[u], i[u]) ? 1 : 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int r = __reduce_add_sync(kFull, c[u]);
                    if (lane == 0 && i[u] != 0xFFFFFFFFu && r == k - 1) {
                        s_t2d = d[u];  // a single warp can reach this
                        s_t2i = i[u];
                    }
                }
            }
        } else {
            for (int L = tid - 32 * w0; L < nlists; L += 32 * nr) {
                const float d = ld[L * k];
                const uint32_t i = lid[L * k];
                if (i == 0xFFFFFFFFu) continue;
                int r = 0;
#pragma unroll 8
                for (int M = 0; M < nlists; ++M) r += better(ld[M * k], lid[M * k], d, i) ? 1 : 0;
                if (r == k - 1) {
                    s_t2d = d;  // a single thread can reach this
                    s_t2i = i;
                }
            }
        }
    }
    __syncthreads();
    td_out = s_td;
    ti_out = s_ti;
    if (better(s_t2d, s_t2i, td_out, ti_out)) {
        td_out = s_t2d;
        ti_out = s_t2i;
    }
}

// The k best of `nlists` sorted lists of k entries each (list L at [L*k,
// L*k+k), padding (+inf, UINT32_MAX) at its end), written ascending to
// od / oi (shared or global), padded when fewer exist. Threshold filter +
// rank counting (see the file comment); returns false, having written
// nothing, when more than kSelCap entries survive the threshold. Block-wide;
// the caller synchronises before reusing ld / lid / sv_*.
__device__ inline bool block_select(const float* ld, const uint32_t* lid, int nlists, int k, float* sv_d, uint32_t* sv_id,
                             float* od, uint32_t* oi) {
    __shared__ int s_n;
    const int tid = threadIdx.x, nt = blockDim.x;
    float td;
    uint32_t ti;
    if (tid == 0) s_n = 0;
    lists_threshold(ld, lid, nlists, k, td, ti);
    const int total = nlists * k;
    for (int e = tid; e < total; e += nt) {
        const uint32_t i = lid[e];
        if (i == 0xFFFFFFFFu) continue;
        const float d = ld[e];
        if (better(td, ti, d, i)) continue;  // worse than the threshold
        const int pos = atomicAdd(&s_n, 1);
        if (pos < kSelCap) {
            sv_d[pos] = d;
            sv_id[pos] = i;
        }
    }
    __syncthreads();
    const int S = s_n;
    if (S > kSelCap) return false;
    for (int s = tid; s < S; s += nt) {
        const float d = sv_d[s];
        const uint32_t i = sv_id[s];
        int r = 0;
#pragma unroll 8
        for (int j = 0; j < S; ++j) r += better(sv_d[j], sv_id[j], d, i) ? 1 : 0;
        if (r < k) {
            od[r] = d;
            oi[r] = i;
        }
    }
    for (int r = S + tid; r < k; r += nt) {
        od[r] = inf_f();
        oi[r] = 0xFFFFFFFFu;
    }
    return true;
}

// block_select over lists that other CTAs wrote to global memory (read
// through L2): list L's entries at [L*stride, L*stride + k).
__device__ inline bool block_select_g(const float* ld, const uint32_t* lid, int nlists, int stride, int k,
                                      float* sv_d, uint32_t* sv_id, float* od, uint32_t* oi) {
    __shared__ float s_td;
    __shared__ uint32_t s_ti;
    __shared__ int s_n;
    const int tid = threadIdx.x, lane = tid & 31, nt = blockDim.x;
    if (tid < 32) {
        float td = inf_f();
        uint32_t ti = 0xFFFFFFFFu;
        for (int L = lane; L < nlists; L += 32) {
            const float d = __ldcg(ld + static_cast<size_t>(L) * stride + k - 1);
            const uint32_t i = __ldcg(lid + static_cast<size_t>(L) * stride + k - 1);
            if (better(d, i, td, ti)) { td = d; ti = i; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float d = __shfl_xor_sync(kFull, td, o);
            const uint32_t i = __shfl_xor_sync(kFull, ti, o);
            if (better(d, i, td, ti)) { td = d; ti = i; }
        }
        if (lane == 0) {
            s_td = td;
            s_ti = ti;
            s_n = 0;
        }
    }
    __syncthreads();
    const float td = s_td;
    const uint32_t ti = s_ti;
    for (int e = tid; e < nlists * k; e += nt) {
        const int L = e / k, j = e - L * k;
        const uint32_t i = __ldcg(lid + static_cast<size_t>(L) * stride + j);
        if (i == 0xFFFFFFFFu) continue;
        const float d = __ldcg(ld + static_cast<size_t>(L) * stride + j);
        if (better(td, ti, d, i)) continue;
        const int pos = atomicAdd(&s_n, 1);
        if (pos < kSelCap) {
            sv_d[pos] = d;
            sv_id[pos] = i;
        }
    }
    __syncthreads();
    const int S = s_n;
    if (S > kSelCap) return false;
    for (int s = tid; s < S; s += nt) {
        const float d = sv_d[s];
        const uint32_t i = sv_id[s];
        int r = 0;
#pragma unroll 8
        for (int j = 0; j < S; ++j) r += better(sv_d[j], sv_id[j], d, i) ? 1 : 0;
        if (r < k) {
            od[r] = d;
            oi[r] = i;
        }
    }
    for (int r = S + tid; r < k; r += nt) {
        od[r] = inf_f();
        oi[r] = 0xFFFFFFFFu;
    }
    return true;
}

// Bitonic fallback of block_select: sort all nlists*k entries in place
// (sd / si hold at least next_pow2(nlists*k) entries) and copy the first k.
__device__ inline void block_sort_select(float* sd, uint32_t* si, int nlists, int k, float* od, uint32_t* oi) {
    const int n = nlists * k, pn = next_pow2(n);
    for (int i = n + threadIdx.x; i < pn; i += blockDim.x) {
        sd[i] = inf_f();
        si[i] = 0xFFFFFFFFu;
    }
    __syncthreads();
    block_bitonic_sort(sd, si, pn);
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        od[j] = sd[j];
        oi[j] = si[j];
    }
}

}  // namespace scan1
}  // namespace e8qc
