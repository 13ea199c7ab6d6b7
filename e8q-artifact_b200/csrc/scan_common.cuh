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
constexpr int kSelCap = 256;      // survivors of a threshold select (counted or sorted)
constexpr int kSelCapWide = 1024;  // the same for the pruned search's seed selects

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

// Entry j of list L: shared memory, or global memory written by other CTAs
// (read through L2).
template <bool G>
__device__ __forceinline__ float lst_d(const float* ld, size_t e) {
    if constexpr (G) return __ldcg(ld + e);
    else return ld[e];
}
template <bool G>
__device__ __forceinline__ uint32_t lst_i(const uint32_t* lid, size_t e) {
    if constexpr (G) return __ldcg(lid + e);
    else return lid[e];
}

// The sharper of two upper bounds of the k-th best entry of `nlists` sorted
// lists of k entries each (list L's entries at [L*stride, L*stride + k)):
// the best of the lists' k-th entries (that list holds k entries at or below
// it), and T_m = the need-th best of the lists' m-th entries, m = ceil(k /
// nlists), need = ceil(k / m) <= nlists (`need` lists each hold m entries at
// or below it: need * m >= k; with nlists >= k this is the k-th best head).
// Warp 0 forms the first; the other warps the second, each holding the lists'
// m-th entries in registers (lane l: lists l, l + 32, ...) and ranking four of
// its share per step with a warp reduction. Block-wide (all threads call; the
// result is in every thread).
template <bool G>
__device__ inline void lists_threshold_t(const float* ld, const uint32_t* lid, int nlists, int stride, int k,
                                         float& td_out, uint32_t& ti_out) {
    __shared__ float s_td, s_t2d;
    __shared__ uint32_t s_ti, s_t2i;
    const int tid = threadIdx.x, lane = tid & 31, nt = blockDim.x;
    const int warp = tid >> 5, nw = nt >> 5;
    if (tid == 0) {
        s_t2d = inf_f();
        s_t2i = 0xFFFFFFFFu;
    }
    __syncthreads();
    if (warp == 0) {
        float td = inf_f();
        uint32_t ti = 0xFFFFFFFFu;
#pragma unroll 8
        for (int L = lane; L < nlists; L += 32) {
            const size_t e = static_cast<size_t>(L) * stride + k - 1;
            const float d = lst_d<G>(ld, e);
            const uint32_t i = lst_i<G>(lid, e);
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
    constexpr int kHpl = 8;  // entries per lane: up to 256 lists
    const int m = nlists > 0 ? (k + nlists - 1) / nlists : 1;
    const int need = (k + m - 1) / m;
    const int w0 = nw > 1 ? 1 : 0, nr = nw - w0;
    if (nlists > 0 && nlists <= 32 * kHpl && warp >= w0) {
        float hd[kHpl];
        uint32_t hi[kHpl];
#pragma unroll
        for (int u = 0; u < kHpl; ++u) {
            const int L = lane + 32 * u;
            const size_t e = static_cast<size_t>(L) * stride + m - 1;
            hd[u] = L < nlists ? lst_d<G>(ld, e) : inf_f();
            hi[u] = L < nlists ? lst_i<G>(lid, e) : 0xFFFFFFFFu;
        }
        for (int L0 = warp - w0; L0 < nlists; L0 += 4 * nr) {
            int c[4] = {0, 0, 0, 0};
            float d[4];
            uint32_t i[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int L = L0 + u * nr;
                const size_t e = static_cast<size_t>(L) * stride + m - 1;
                d[u] = L < nlists ? lst_d<G>(ld, e) : inf_f();
                i[u] = L < nlists ? lst_i<G>(lid, e) : 0xFFFFFFFFu;
            }
#pragma unroll
            for (int u2 = 0; u2 < kHpl; ++u2)
#pragma unroll
                for (int u = 0; u < 4; ++u) c[u] += better(hd[u2], hi[u2], d[u], i[u]) ? 1 : 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int r = __reduce_add_sync(kFull, c[u]);
                // real entries are unique; padding only matters when fewer
                // than `need` lists hold m real entries
                if (lane == 0 && i[u] != 0xFFFFFFFFu && r == need - 1) {
                    s_t2d = d[u];  // a single warp can reach this
                    s_t2i = i[u];
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

__device__ inline void lists_threshold(const float* ld, const uint32_t* lid, int nlists, int k, float& td_out,
                                       uint32_t& ti_out) {
    lists_threshold_t<false>(ld, lid, nlists, k, k, td_out, ti_out);
}

// The entries at or below the threshold (td, ti), compacted into sv_* with
// one shared atomic per warp and step (lanes' slots from a ballot), then the
// k best of them written ascending to od / oi: ranked by counting when few
// survive, else sorted (a block bitonic sort of at most `cap` entries).
// False, having written nothing, when more than `cap` (sv_*'s size) survive.
template <bool G>
__device__ inline bool filter_select(const float* ld, const uint32_t* lid, int nlists, int stride, int k, float td,
                                     uint32_t ti, int* s_n, float* sv_d, uint32_t* sv_id, float* od, uint32_t* oi,
                                     int cap) {
    const int tid = threadIdx.x, lane = tid & 31, nt = blockDim.x;
    const int total = nlists * k;
    if constexpr (!G) {
        // lists in shared memory: one pass, a shared atomic per survivor
        // (few survive the bounds; the short loop keeps the merge's code
        // small)
        for (int e = tid; e < total; e += nt) {
            const uint32_t i = lid[e];
            if (i == 0xFFFFFFFFu) continue;
            const float d = ld[e];
            if (better(td, ti, d, i)) continue;  // worse than the threshold
            const int pos = atomicAdd(s_n, 1);
            if (pos < cap) {
                sv_d[pos] = d;
                sv_id[pos] = i;
            }
        }
    }
    // lists in global memory: eight entries per thread per round, loaded
    // before any is filtered (one memory latency per round)
    constexpr int kPer = 8;
    for (int b0 = 0; G && b0 < total; b0 += kPer * nt) {  // the same trip count in every thread
        float d[kPer];
        uint32_t i[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int e = b0 + u * nt + tid;
            d[u] = 0.0f;
            i[u] = 0xFFFFFFFFu;
            if (e < total) {
                const int L = e / k, j = e - L * k;
                const size_t a = static_cast<size_t>(L) * stride + j;
                i[u] = lst_i<G>(lid, a);
                d[u] = lst_d<G>(ld, a);
            }
        }
        // the round's masks first (independent votes), then one shared
        // atomic per warp and round, only when something survives
        unsigned mk[kPer];
        bool keep[kPer];
        int tot = 0;
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            keep[u] = i[u] != 0xFFFFFFFFu && !better(td, ti, d[u], i[u]);  // not worse than the threshold
            mk[u] = __ballot_sync(kFull, keep[u]);
            tot += __popc(mk[u]);
        }
        if (tot != 0) {  // warp-uniform
            int wb = 0;
            if (lane == 0) wb = atomicAdd(s_n, tot);
            wb = __shfl_sync(kFull, wb, 0);
            const unsigned below = (1u << lane) - 1u;
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                if (keep[u]) {
                    const int pos = wb + __popc(mk[u] & below);
                    if (pos < cap) {
                        sv_d[pos] = d[u];
                        sv_id[pos] = i[u];
                    }
                }
                wb += __popc(mk[u]);
            }
        }
    }
    __syncthreads();
    const int S = *s_n;
    if (S > cap) return false;
    if (S <= 64) {
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
    const int pn = next_pow2(S);
    for (int e = S + tid; e < pn; e += nt) {
        sv_d[e] = inf_f();
        sv_id[e] = 0xFFFFFFFFu;
    }
    __syncthreads();
    block_bitonic_sort(sv_d, sv_id, pn);
    for (int r = tid; r < k; r += nt) {
        od[r] = r < S ? sv_d[r] : inf_f();
        oi[r] = r < S ? sv_id[r] : 0xFFFFFFFFu;
    }
    return true;
}

// The selects below are not inlined: a kernel calls them at several sites,
// once each per launch, and one shared copy of their code stays warm in the
// instruction cache where inlined copies would each be fetched cold.
//
// The k best of `nlists` sorted lists of k entries each (list L at [L*k,
// L*k+k), padding (+inf, UINT32_MAX) at its end), written ascending to
// od / oi (shared or global), padded when fewer exist. Threshold filter +
// rank counting or a survivors' sort (see the file comment); returns false,
// having written nothing, when more than kSelCap entries survive the
// threshold. Block-wide; the caller synchronises before reusing ld / lid /
// sv_*.
static __device__ __noinline__ bool block_select(const float* ld, const uint32_t* lid, int nlists, int k, float* sv_d, uint32_t* sv_id,
                             float* od, uint32_t* oi, int cap = kSelCap) {
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    float td;
    uint32_t ti;
    lists_threshold(ld, lid, nlists, k, td, ti);
    return filter_select<false>(ld, lid, nlists, k, k, td, ti, &s_n, sv_d, sv_id, od, oi, cap);
}

// block_select over lists that other CTAs wrote to global memory (read
// through L2): list L's entries at [L*stride, L*stride + k).
static __device__ __noinline__ bool block_select_g(const float* ld, const uint32_t* lid, int nlists, int stride, int k,
                                      float* sv_d, uint32_t* sv_id, float* od, uint32_t* oi, int cap = kSelCap) {
    __shared__ int s_n;
    if (threadIdx.x == 0) s_n = 0;
    float td;
    uint32_t ti;
    lists_threshold_t<true>(ld, lid, nlists, stride, k, td, ti);
    return filter_select<true>(ld, lid, nlists, stride, k, td, ti, &s_n, sv_d, sv_id, od, oi, cap);
}


// Bitonic fallback of block_select: sort all nlists*k entries in place
// (sd / si hold at least next_pow2(nlists*k) entries) and copy the first k.
static __device__ __noinline__ void block_sort_select(float* sd, uint32_t* si, int nlists, int k, float* od, uint32_t* oi) {
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
