// Search-path kernels: query rotation, one-query routing with on-device
// top-nprobe selection, and the single-vector estimator. (The plain scan is
// in scan_plain.cu, the batched path in batched.cu.)
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "device_common.cuh"
#include "internal.h"
#include "tma.cuh"

namespace e8qc {

namespace {

// Block-wide exclusive scan of one int per thread (blockDim <= 1024).
__device__ int block_exclusive_scan(int v, int* total, int* sm32) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm32[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = lane < nw ? sm32[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, s, o);
            if (lane >= o) s += y;
        }
        sm32[lane] = s;
    }
    __syncthreads();
    const int before = (warp > 0 ? sm32[warp - 1] : 0) + x - v;
    *total = sm32[nw - 1];
    __syncthreads();
    return before;
}

// The same over 64-bit values (two packed 32-bit counts whose sums stay
// below 2^32 add without carries).
__device__ unsigned long long block_exclusive_scan64(unsigned long long v, unsigned long long* total,
                                                     unsigned long long* sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long t = lane < nw ? sm[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, t, o);
            if (lane >= o) t += y;
        }
        sm[lane] = t;
    }
    __syncthreads();
    const unsigned long long before = (warp > 0 ? sm[warp - 1] : 0ull) + x - v;
    *total = sm[nw - 1];
    __syncthreads();
    return before;
}

// ---------------------------------------------------------------------------
// Query rotation: one CTA per query. out = rot(q) - mean_rot.
__global__ void rotate_queries_kernel(const float* __restrict__ q, int dim, int pd, int td,
                                      float fac, const uint8_t* __restrict__ signs,
                                      const float* __restrict__ subtract, float* __restrict__ out) {
    extern __shared__ float sx[];
    const size_t row = blockIdx.x;
    for (int i = threadIdx.x; i < pd; i += blockDim.x) sx[i] = i < dim ? q[row * dim + i] : 0.0f;
    __syncthreads();
    rotate_rows_smem(sx, 1, pd, pd, td, fac, signs);
    for (int i = threadIdx.x; i < pd; i += blockDim.x)
        out[row * pd + i] = subtract ? __fsub_rn(sx[i], subtract[i]) : sx[i];
}

// Register form of the same rotation for padded_dim <= 1024: one warp per
// row, lane l holding elements j*32 + l (j < NJ = padded_dim / 32) in
// registers. Butterfly stages with h < 32 exchange values between lanes
// (shfl_xor h), stages with h >= 32 pair registers j and j + h/32 of a lane;
// the stages, their order and every rounding are those of rotate_rows_smem
// (sign flip over the whole row, FHT of size td at offset 0 or
// padded_dim - td alternately, scale by fac, Kac half-swap when td <
// padded_dim, final 0.25 when padded), so the two forms agree bit for bit.
template <int NJ, int J0, int TJ>
__device__ __forceinline__ void fht_scale_regs(float (&v)[NJ], int lane, float fac) {
#pragma unroll
    for (int h = 1; h < 32; h <<= 1) {
        const bool lower = (lane & h) == 0;
#pragma unroll
        for (int j = J0; j < J0 + TJ; ++j) {
            const float o = __shfl_xor_sync(kFull, v[j], h);
            v[j] = lower ? __fadd_rn(v[j], o) : __fsub_rn(o, v[j]);
        }
    }
#pragma unroll
    for (int H = 1; H < TJ; H <<= 1) {
#pragma unroll
        for (int j = J0; j < J0 + TJ; ++j) {
            if (((j - J0) & H) == 0) {
                const float a0 = v[j], a1 = v[j + H];
                v[j] = __fadd_rn(a0, a1);
                v[j + H] = __fsub_rn(a0, a1);
            }
        }
    }
#pragma unroll
    for (int j = J0; j < J0 + TJ; ++j) v[j] = __fmul_rn(v[j], fac);
}

constexpr int kRotWarps = 4;  // rows per CTA of the register form

template <int NJ, int TJ>
__global__ void __launch_bounds__(kRotWarps * 32) rotate_rows_warp_kernel(
    const float* __restrict__ q, int dim, int n, float fac, const uint8_t* __restrict__ signs,
    const float* __restrict__ subtract, float* __restrict__ out) {
    constexpr int PD = NJ * 32;
    constexpr bool kPadded = TJ != NJ;
    const int lane = threadIdx.x & 31;
    const size_t row = static_cast<size_t>(blockIdx.x) * kRotWarps + (threadIdx.x >> 5);
    if (row >= static_cast<size_t>(n)) return;
    float v[NJ];
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
        const int i = j * 32 + lane;
        v[j] = i < dim ? q[row * dim + i] : 0.0f;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        // sign bit of element j*32 + l = bit l of the round's little-endian word j
        const uint32_t* sw = reinterpret_cast<const uint32_t*>(signs + r * (PD / 8));
#pragma unroll
        for (int j = 0; j < NJ; ++j)
            if ((__ldg(sw + j) >> lane) & 1u) v[j] = -v[j];
        if (!kPadded || (r & 1) == 0)
            fht_scale_regs<NJ, 0, TJ>(v, lane, fac);
        else
            fht_scale_regs<NJ, NJ - TJ, TJ>(v, lane, fac);
        if (kPadded) {
#pragma unroll
            for (int j = 0; j < NJ / 2; ++j) {
                const float a0 = v[j], a1 = v[j + NJ / 2];
                v[j] = __fadd_rn(a0, a1);
                v[j + NJ / 2] = __fsub_rn(a0, a1);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
        const int i = j * 32 + lane;
        const float x = kPadded ? __fmul_rn(v[j], 0.25f) : v[j];
        out[row * PD + i] = subtract ? __fsub_rn(x, subtract[i]) : x;
    }
}

constexpr int largest_pow2_le(int x) { return x >= 2 ? 2 * largest_pow2_le(x / 2) : 1; }

template <int NJ>
bool launch_rotate_warp_nj(int tj, const float* q, int dim, int n, float fac, const uint8_t* signs,
                           const float* subtract, float* out, cudaStream_t s) {
    constexpr int P = largest_pow2_le(NJ);
    const unsigned grid = static_cast<unsigned>((n + kRotWarps - 1) / kRotWarps);
    if (tj == P)
        rotate_rows_warp_kernel<NJ, P><<<grid, kRotWarps * 32, 0, s>>>(q, dim, n, fac, signs, subtract, out);
    else if (P >= 2 && tj == P / 2)
        rotate_rows_warp_kernel<NJ, (P >= 2 ? P / 2 : 1)><<<grid, kRotWarps * 32, 0, s>>>(q, dim, n, fac, signs,
                                                                                         subtract, out);
    else
        return false;
    return true;
}

// Register-form rotation when it applies (padded_dim <= 1024, td >= 32,
// 4-byte aligned sign rounds); false leaves the row to the shared-memory form.
bool launch_rotate_warp(int dim, int pd, int td, const float* q, int n, float fac, const uint8_t* signs,
                        const float* subtract, float* out, cudaStream_t s) {
    if (n <= 0 || pd % 64 != 0 || pd > 1024 || td < 32 || (reinterpret_cast<uintptr_t>(signs) & 3u) != 0)
        return false;
    const int tj = td / 32;
    switch (pd / 32) {
#define E8QC_ROT_CASE(NJ) \
    case NJ:              \
        return launch_rotate_warp_nj<NJ>(tj, q, dim, n, fac, signs, subtract, out, s);
        E8QC_ROT_CASE(2) E8QC_ROT_CASE(4) E8QC_ROT_CASE(6) E8QC_ROT_CASE(8) E8QC_ROT_CASE(10) E8QC_ROT_CASE(12)
        E8QC_ROT_CASE(14) E8QC_ROT_CASE(16) E8QC_ROT_CASE(18) E8QC_ROT_CASE(20) E8QC_ROT_CASE(22)
        E8QC_ROT_CASE(24) E8QC_ROT_CASE(26) E8QC_ROT_CASE(28) E8QC_ROT_CASE(30) E8QC_ROT_CASE(32)
#undef E8QC_ROT_CASE
        default:
            return false;
    }
}

// ---------------------------------------------------------------------------
// Top-nprobe lists of one query by 64-bit key (float bits of d2 << 32 | cid),
// src/index/ivf_route.cpp:9-27 + src/simd/kernels.hpp:13-21. Keys are unique,
// so an MSB radix select finds the nprobe-th key exactly; the selected lists
// are compacted in cid order (the plain scan's result does not depend on
// probe order) with their first tile and length, and the tile-count prefix.
//
// select_probes_reg: up to kRegKeys keys per thread, held in registers (thread
// t holds keys [t * kpt, t * kpt + kpt), kpt = ceil(nlist / blockDim)); the
// lists' first tiles and lengths are staged in shared memory (stb: nlist + 1,
// slen: nlist) beside them, and compaction and tile prefix are one block
// scan of each thread's (selected lists, their tiles). The nprobe-th key is
// found by one bucket pass: 256 buckets over [min d2, max d2] (a monotone map
// of d2, so every key of a lower bucket is smaller than every key of a
// higher one); the keys of the bucket holding the nprobe-th are gathered and
// ranked by counting. When that bucket holds more than kBucketCap keys (d2
// values piled up, or not finite) an MSB radix select over the registers
// takes over: each 8-bit pass histograms the keys that still match the
// prefix with one shared atomic per distinct bin per warp (lanes with equal
// bins found by __match_any_sync); the cid half of a key is below 2^16, so
// its two top bytes need no pass.
constexpr int kRegKeys = 16;
constexpr int kBucketCap = 256;

// Warp 0 finds the bin holding the s_want-th key of the histogram and
// narrows the prefix (shared by both selects).
__device__ __forceinline__ void radix_pick(const int* hist, uint64_t prefix, int shift, uint64_t* s_prefix,
                                           int* s_want) {
    const int lane = threadIdx.x;
    int cnt[8], tot = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        cnt[j] = hist[lane * 8 + j];
        tot += cnt[j];
    }
    int incl = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    const int excl = incl - tot;
    const int want = *s_want;
    const unsigned hit = __ballot_sync(kFull, excl < want && incl >= want);
    const int owner = __ffs(hit) - 1;
    if (lane == owner) {
        int cum = excl, sel = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (cum + cnt[j] >= want) {
                sel = j;
                break;
            }
            cum += cnt[j];
        }
        *s_prefix = prefix | (static_cast<uint64_t>(lane * 8 + sel) << shift);
        *s_want = want - cum;
    }
}

__device__ void select_probes_reg(const DevIndex& ix, const uint64_t* gkeys, int nprobe, const RouteWork& w,
                                  uint32_t* stb, uint32_t* slen) {
    __shared__ int hist[256];
    __shared__ uint64_t s_prefix;
    __shared__ int s_want;
    __shared__ uint32_t s_lo[32], s_hi[32];
    __shared__ int s_bucket, s_nb, s_nc;
    __shared__ bool s_done;
    __shared__ unsigned long long s_cand[kBucketCap];
    __shared__ unsigned long long sm64[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x, nw = nt >> 5;
    const int nlist = ix.nlist;
    const int kpt = (nlist + nt - 1) / nt;  // keys per thread (<= kRegKeys)
    nprobe = nprobe < nlist ? nprobe : nlist;
    unsigned long long key[kRegKeys];
    uint32_t lo = 0xFFFFFFFFu, hi = 0u;  // d2 bits (non-negative floats order as integers)
#pragma unroll
    for (int j = 0; j < kRegKeys; ++j) {
        const int c = tid * kpt + j;
        key[j] = (j < kpt && c < nlist) ? __ldcg(reinterpret_cast<const unsigned long long*>(gkeys) + c) : ~0ull;
        if (j < kpt && c < nlist) {
            const uint32_t b = static_cast<uint32_t>(key[j] >> 32);
            lo = min(lo, b);
            hi = max(hi, b);
        }
    }
    for (int c = tid; c < nlist; c += nt) {
        stb[c] = ix.tile_begin[c];
        slen[c] = ix.list_len[c];
    }
    for (int i = tid; i < 256; i += nt) hist[i] = 0;
    lo = __reduce_min_sync(kFull, lo);
    hi = __reduce_max_sync(kFull, hi);
    if (lane == 0) {
        s_lo[warp] = lo;
        s_hi[warp] = hi;
    }
    if (tid == 0) {
        stb[nlist] = ix.tile_begin[nlist];
        s_prefix = 0;
        s_want = nprobe;
        s_nc = 0;
        s_done = false;
    }
    __syncthreads();
    if (tid < 32) {
        lo = lane < nw ? s_lo[lane] : 0xFFFFFFFFu;
        hi = lane < nw ? s_hi[lane] : 0u;
        lo = __reduce_min_sync(kFull, lo);
        hi = __reduce_max_sync(kFull, hi);
        if (lane == 0) {
            s_lo[0] = lo;
            s_hi[0] = hi;
        }
    }
    __syncthreads();
    lo = s_lo[0];
    hi = s_hi[0];
    const float flo = __uint_as_float(lo), fhi = __uint_as_float(hi);
    // d2 is finite and >= 0 when hi < +inf; scale 0 (one bucket) when all equal
    const bool finite = hi < 0x7F800000u;
    const float span = __fsub_rn(fhi, flo);
    const float scale = (finite && span > 1.0e-30f && span < 3.0e38f) ? __fdiv_rn(256.0f, span) : 0.0f;
    auto bucket = [&](unsigned long long kk) {
        const float d = __uint_as_float(static_cast<uint32_t>(kk >> 32));
        const int b = static_cast<int>(__fmul_rn(__fsub_rn(d, flo), scale));
        return b < 255 ? b : 255;
    };
    if (finite) {
#pragma unroll
        for (int j = 0; j < kRegKeys; ++j) {
            if (j >= kpt) break;  // uniform over the block
            if (tid * kpt + j < nlist) atomicAdd(&hist[bucket(key[j])], 1);
        }
    }
    __syncthreads();
    if (finite && tid < 32) {
        // the bucket holding the nprobe-th key
        int cnt[8], tot = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            cnt[j] = hist[lane * 8 + j];
            tot += cnt[j];
        }
        int incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - tot;
        const unsigned hitm = __ballot_sync(kFull, excl < nprobe && incl >= nprobe);
        if (lane == __ffs(hitm) - 1) {
            int cum = excl, sel = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (cum + cnt[j] >= nprobe) {
                    sel = j;
                    break;
                }
                cum += cnt[j];
            }
            s_bucket = lane * 8 + sel;
            s_want = nprobe - cum;
            s_nb = cnt[sel];
        }
    }
    __syncthreads();
    if (finite && s_nb <= kBucketCap) {
        const int bs = s_bucket;
#pragma unroll
        for (int j = 0; j < kRegKeys; ++j) {
            if (j >= kpt) break;
            if (tid * kpt + j < nlist && bucket(key[j]) == bs) s_cand[atomicAdd(&s_nc, 1)] = key[j];
        }
        __syncthreads();
        // the want-th smallest of the bucket's keys, by rank counting
        const int nb = s_nc, want = s_want;
        for (int i = tid; i < nb; i += nt) {
            const unsigned long long x = s_cand[i];
            int r = 0;
#pragma unroll 8
            for (int m = 0; m < nb; ++m) r += s_cand[m] < x ? 1 : 0;
            if (r == want - 1) {
                s_prefix = x;  // keys are unique: one thread
                s_done = true;
            }
        }
        __syncthreads();
    }
    const bool bucket_done = s_done;
    if (!bucket_done && tid == 0) {
        s_prefix = 0;
        s_want = nprobe;
    }
    uint64_t mask = 0;
    for (int shift = 56; shift >= 0 && !bucket_done; shift -= 8) {
        if (shift == 24 || shift == 16) {  // cid bits 16..31: zero in every key
            mask |= 0xFFull << shift;
            continue;
        }
        for (int i = tid; i < 256; i += nt) hist[i] = 0;
        __syncthreads();
        const uint64_t prefix = s_prefix;
#pragma unroll
        for (int j = 0; j < kRegKeys; ++j) {
            if (j >= kpt) break;  // uniform over the block
            const int c = tid * kpt + j;
            const bool in = c < nlist && (key[j] & mask) == prefix;
            // lanes outside the prefix get a bin of their own (>= 256)
            const uint32_t bin = in ? static_cast<uint32_t>((key[j] >> shift) & 255u) : 256u + lane;
            const unsigned m = __match_any_sync(kFull, bin);
            if (in && lane == __ffs(m) - 1) atomicAdd(&hist[bin], __popc(m));
        }
        __syncthreads();
        if (tid < 32) radix_pick(hist, prefix, shift, &s_prefix, &s_want);
        mask |= 0xFFull << shift;
        __syncthreads();
    }
    const uint64_t kth = s_prefix;
    // compact keys <= kth in cid order, with their tile offsets: one scan of
    // (lists, tiles) per thread, then each thread writes its lists in order
    uint32_t cnt = 0, tiles = 0;
#pragma unroll
    for (int j = 0; j < kRegKeys; ++j) {
        const int c = tid * kpt + j;
        if (j < kpt && c < nlist && key[j] <= kth) {
            ++cnt;
            tiles += stb[c + 1] - stb[c];
        }
    }
    unsigned long long tot;
    const unsigned long long before =
        block_exclusive_scan64((static_cast<unsigned long long>(cnt) << 32) | tiles, &tot, sm64);
    uint32_t pos = static_cast<uint32_t>(before >> 32), toff = static_cast<uint32_t>(before);
#pragma unroll
    for (int j = 0; j < kRegKeys; ++j) {
        const int c = tid * kpt + j;
        if (j < kpt && c < nlist && key[j] <= kth) {
            w.probes[pos] = static_cast<uint32_t>(c);
            w.probe_d2[pos] = __uint_as_float(static_cast<uint32_t>(key[j] >> 32));
            w.probe_info[pos] = make_uint2(stb[c], slen[c]);
            w.tile_off[pos] = toff;
            ++pos;
            toff += stb[c + 1] - stb[c];
        }
    }
    if (tid == 0) {
        w.tile_off[nprobe] = static_cast<uint32_t>(tot);
        *w.total_tiles = static_cast<uint32_t>(tot);
    }
}

// select_probes: any nlist; keys in shared memory when they fit (skeys),
// else read through L2 on every pass (8 passes).
__device__ void select_probes(const DevIndex& ix, const uint64_t* gkeys, int nprobe,
                              const RouteWork& w, unsigned long long* skeys) {
    __shared__ int hist[256];
    __shared__ uint64_t s_prefix;
    __shared__ int s_want;
    __shared__ int sm32[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int nlist = ix.nlist;
    nprobe = nprobe < nlist ? nprobe : nlist;
    const unsigned long long* keys = reinterpret_cast<const unsigned long long*>(gkeys);
    if (skeys != nullptr) {
        for (int c = tid; c < nlist; c += nt) skeys[c] = __ldcg(keys + c);
        keys = skeys;
    }
    if (tid == 0) {
        s_prefix = 0;
        s_want = nprobe;
    }
    uint64_t mask = 0;
    __syncthreads();
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += nt) hist[i] = 0;
        __syncthreads();
        const uint64_t prefix = s_prefix;
        for (int c = tid; c < nlist; c += nt) {
            const uint64_t key = skeys ? keys[c] : __ldcg(keys + c);
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1);
        }
        __syncthreads();
        if (tid < 32) radix_pick(hist, prefix, shift, &s_prefix, &s_want);
        mask |= 0xFFull << shift;
        __syncthreads();
    }
    const uint64_t kth = s_prefix;
    // compact keys <= kth in cid order
    int base = 0;
    for (int c0 = 0; c0 < nlist; c0 += nt) {
        const int c = c0 + tid;
        uint64_t key = ~0ull;
        if (c < nlist) key = skeys ? keys[c] : __ldcg(keys + c);
        const int flag = (c < nlist && key <= kth) ? 1 : 0;
        int tot;
        const int pos = base + block_exclusive_scan(flag, &tot, sm32);
        if (flag) {
            w.probes[pos] = static_cast<uint32_t>(c);
            w.probe_d2[pos] = __uint_as_float(static_cast<uint32_t>(key >> 32));
        }
        base += tot;
    }
    __syncthreads();
    // tile prefix, first tile and length of the probed lists
    int tbase = 0;
    for (int p0 = 0; p0 < nprobe; p0 += nt) {
        const int p = p0 + tid;
        int t = 0;
        if (p < nprobe) {
            const uint32_t c = __ldcg(w.probes + p);
            const uint32_t tb = ix.tile_begin[c];
            t = static_cast<int>(ix.tile_begin[c + 1] - tb);
            w.probe_info[p] = make_uint2(tb, ix.list_len[c]);
        }
        int tot;
        const int pos = tbase + block_exclusive_scan(t, &tot, sm32);
        if (p < nprobe) w.tile_off[p] = static_cast<uint32_t>(pos);
        tbase += tot;
    }
    if (tid == 0) {
        w.tile_off[nprobe] = static_cast<uint32_t>(tbase);
        *w.total_tiles = static_cast<uint32_t>(tbase);
    }
}

// d2 of one rotated query to every centroid (fp32 products summed in fp64,
// as the scalar GEMV src/simd/kernels_generic.cpp:13-33), then the last CTA
// to finish selects the probes.
__global__ void route_one_kernel(DevIndex ix, const float* __restrict__ rq, int nprobe,
                                 RouteWork w, unsigned s_dyn_bytes) {
    extern __shared__ __align__(16) float sq[];
    __shared__ double red[32];
    __shared__ float s_qn2;
    __shared__ bool s_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    // the scan launched after this one may start its own setup now
    launch_dependents();
    const int pd = ix.pd;
    double part = 0.0;
    for (int i = tid; i < pd; i += blockDim.x) {
        const float v = rq[i];
        sq[i] = v;
        part += static_cast<double>(v) * static_cast<double>(v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    if (lane == 0) red[warp] = part;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int i = 0; i < nw; ++i) s += red[i];
        s_qn2 = static_cast<float>(s);
    }
    __syncthreads();
    const float qn2 = s_qn2;
    // one centroid per warp iteration; each lane loads its float4s of the row
    // first (one memory latency per row), then accumulates in fp64
    for (int c = blockIdx.x * nw + warp; c < ix.nlist; c += gridDim.x * nw) {
        const float4* cc = reinterpret_cast<const float4*>(ix.cen + static_cast<size_t>(c) * pd);
        const float4* q4 = reinterpret_cast<const float4*>(sq);
        const int n4 = pd >> 2;
        double dot = 0.0;
        for (int base = 0; base < n4; base += 8 * 32) {
            float4 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int i = base + j * 32 + lane;
                v[j] = i < n4 ? __ldg(cc + i) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int i = base + j * 32 + lane;
                if (i < n4) {
                    const float4 qv = q4[i];
                    dot += static_cast<double>(qv.x) * static_cast<double>(v[j].x);
                    dot += static_cast<double>(qv.y) * static_cast<double>(v[j].y);
                    dot += static_cast<double>(qv.z) * static_cast<double>(v[j].z);
                    dot += static_cast<double>(qv.w) * static_cast<double>(v[j].w);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(kFull, dot, o);
        if (lane == 0) {
            float d2 = __fmaf_rn(-2.0f, static_cast<float>(dot), __fadd_rn(qn2, ix.cn2[c]));
            if (d2 < 0.0f) d2 = 0.0f;
            w.keys[c] = (static_cast<uint64_t>(__float_as_uint(d2)) << 32) | static_cast<uint32_t>(c);
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(w.counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the dynamic shared buffer (query, then free): the lists' first tiles
    // and lengths for the register select, else the keys if they fit
    const int nl = ix.nlist;
    __syncthreads();
    if (nl <= kRegKeys * static_cast<int>(blockDim.x) && static_cast<size_t>(2 * nl + 8) * 4 <= s_dyn_bytes) {
        uint32_t* stb = reinterpret_cast<uint32_t*>(sq);
        select_probes_reg(ix, w.keys, nprobe, w, stb, stb + nl + 4);
    } else {
        unsigned long long* skeys =
            (static_cast<size_t>(nl) * 8 <= s_dyn_bytes) ? reinterpret_cast<unsigned long long*>(sq) : nullptr;
        select_probes(ix, w.keys, nprobe, w, skeys);
    }
    if (tid == 0) *w.counter = 0;
}

// One stored vector: Estimate() of src/index/e8q_oracle.cpp:58-101 (fp32
// qn2/dot chains fused as the reference build fuses them, fp64 score).
template <int BITS>
__global__ void estimate_kernel(DevIndex ix, const float* __restrict__ rq, int list, uint32_t slot,
                                float* __restrict__ out) {
    if (threadIdx.x != 0) return;
    const float* cc = ix.cen + static_cast<size_t>(list) * ix.pd;
    float qn2 = 0.0f, dot = 0.0f;
    for (int i = 0; i < ix.pd; ++i) {
        qn2 = __fmaf_rn(rq[i], rq[i], qn2);
        dot = __fmaf_rn(rq[i], cc[i], dot);
    }
    float d2 = __fmaf_rn(-2.0f, dot, __fadd_rn(qn2, ix.cn2[list]));
    if (d2 < 0.0f) d2 = 0.0f;
    const uint4* tile = ix.codes + static_cast<size_t>(slot / 32) * ix.nch * 32;
    const int lane = slot % 32;
    constexpr int Q = 1 << BITS;
    double acc = 0.0;
    for (int blk = 0; blk < ix.B; ++blk) {
        // gather the block's bits (8*BITS <= 104) from its chunks
        const int off = blk * 8 * BITS;
        uint32_t words[5];
        for (int j = 0; j < 5; ++j) {
            const int wi = (off >> 5) + j;
            const int c = wi >> 2;
            if (c < ix.nch) {
                const uint4 v = tile[c * 32 + lane];
                const uint32_t arr[4] = {v.x, v.y, v.z, v.w};
                words[j] = arr[wi & 3];
            } else {
                words[j] = 0;
            }
        }
        uint32_t dg[8];
        const int br = decode_block<BITS>(words, off & 31, dg);
        for (int i = 0; i < 8; ++i)
            acc += static_cast<double>(rq[blk * 8 + i]) *
                   static_cast<double>(ix.tab[br * Q + static_cast<int>(dg[i])]);
    }
    const float S = static_cast<float>(acc);
    const size_t s = slot;
    *out = __fmaf_rn(-__fmul_rn(2.0f, ix.g1[s]), S, __fadd_rn(d2, ix.h3[s]));
}

// ProbeBoundW (src/index/e8q_oracle.cpp:103-218), one warp per (query,
// stored vector) pair, every term in fp64: the rotated, centred query and the
// vector's raw row against the list centroid (d2, the residual's norm and
// direction), the exact reconstruction (levels / sqrt(Dpad)) and the scan
// basis (class means, `mid`: 2 per digit position) of the stored code, and the
// normalised discrepancy of the zero-parallel-residual bound. The digits are
// those the reference's 8-bit split decoder returns (e8q_scan.cpp:34-60 as
// called there): at 1 bit digit 7 reads the branch and the branch reads 0; at
// 9 bits and up each digit keeps its low 8 bits. Sums run per lane, then a
// warp reduction (the reference sums in dimension order: results agree to
// ~1e-12 relative).
template <int BITS>
__global__ void probe_bound_kernel(DevIndex ix, const float* __restrict__ rq, const float* __restrict__ rx,
                                   const uint32_t* __restrict__ qsel, const uint32_t* __restrict__ slot_of,
                                   const uint32_t* __restrict__ list_of, const double* __restrict__ dlev,
                                   const double* __restrict__ mid, int m, int dim, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int pair = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (pair >= m) return;
    const double qnan = __longlong_as_double(0x7ff8000000000000ll);
    const uint32_t slot = slot_of[pair];
    if (slot == 0xFFFFFFFFu) {
        if (lane == 0) out[pair] = qnan;
        return;
    }
    const int pd = ix.pd;
    const float* cc = ix.cen + static_cast<size_t>(list_of[pair]) * pd;
    const float* q = rq + static_cast<size_t>(qsel[pair]) * pd;
    const float* xr = rx + static_cast<size_t>(pair) * pd;
    auto wsum = [](double v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
        return v;
    };
    double d2 = 0.0, rn2 = 0.0;
    for (int d = lane; d < pd; d += 32) {
        const double a = static_cast<double>(q[d]) - static_cast<double>(cc[d]);
        const double b = static_cast<double>(xr[d]) - static_cast<double>(cc[d]);
        d2 += a * a;
        rn2 += b * b;
    }
    d2 = wsum(d2);
    rn2 = wsum(rn2);
    const double rn = sqrt(rn2);
    if (!(rn > 0.0)) {
        if (lane == 0) out[pair] = qnan;
        return;
    }
    constexpr int Q = 1 << BITS;
    const uint4* tile = ix.codes + static_cast<size_t>(slot / 32) * ix.nch * 32;
    const int vl = static_cast<int>(slot % 32);
    double dot_ue = 0, n2_e = 0, dot_ce = 0, dot_ew = 0, dot_uw = 0, n2_w = 0, dot_cw = 0, s_exact = 0,
           s_coarse = 0;
    for (int blk = lane; blk < ix.B; blk += 32) {
        const int off = blk * 8 * BITS;
        uint32_t words[5];
        for (int j = 0; j < 5; ++j) {
            const int wi = (off >> 5) + j;
            const int c = wi >> 2;
            if (c < ix.nch) {
                const uint4 v = tile[c * 32 + vl];
                const uint32_t arr[4] = {v.x, v.y, v.z, v.w};
                words[j] = arr[wi & 3];
            } else {
                words[j] = 0;
            }
        }
        uint32_t dg[8];
        int br = decode_block<BITS>(words, off & 31, dg);
        if (BITS == 1) {
            dg[7] = static_cast<uint32_t>(br);
            br = 0;
        } else if (BITS >= 9) {
#pragma unroll
            for (int k = 0; k < 8; ++k) dg[k] &= 0xFFu;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int idx = blk * 8 + k;
            const double ve = dlev[br * Q + static_cast<int>(dg[k])];
            const double wc = mid[2 * k + static_cast<int>(dg[k] >> (BITS - 1))];
            const double c0 = static_cast<double>(cc[idx]);
            const double u = (static_cast<double>(xr[idx]) - c0) / rn;
            dot_ue += u * ve;
            n2_e += ve * ve;
            dot_ce += c0 * ve;
            dot_ew += ve * wc;
            dot_uw += u * wc;
            n2_w += wc * wc;
            dot_cw += c0 * wc;
            s_exact += static_cast<double>(q[idx]) * ve;
            s_coarse += static_cast<double>(q[idx]) * wc;
        }
    }
    dot_ue = wsum(dot_ue);
    n2_e = wsum(n2_e);
    dot_ce = wsum(dot_ce);
    dot_ew = wsum(dot_ew);
    dot_uw = wsum(dot_uw);
    n2_w = wsum(n2_w);
    dot_cw = wsum(dot_cw);
    s_exact = wsum(s_exact);
    s_coarse = wsum(s_coarse);
    if (lane != 0) return;
    double r = qnan;
    if (fabs(dot_ue) > 0.0 && fabs(dot_uw) > 0.0) {
        const double g1 = rn / dot_ue;
        const double h3 = rn2 + 2.0 * g1 * dot_ce;
        const double d_full = d2 + h3 - 2.0 * g1 * s_exact;
        const double w_x = 2.0 * rn / dot_uw;
        const double d_coarse = d2 + rn2 + w_x * dot_cw - w_x * s_coarse;
        const double rx2 = 4.0 * g1 * g1 * n2_e + w_x * w_x * n2_w - 4.0 * g1 * w_x * dot_ew;
        const double omega = sqrt(rx2 > 0.0 ? rx2 : 0.0) / sqrt(static_cast<double>(dim > 1 ? dim - 1 : 1));
        const double r_q = sqrt(d2 > 0.0 ? d2 : 0.0);
        if (omega > 0.0 && r_q > 0.0) r = (d_coarse - d_full) / (r_q * omega);
    }
    out[pair] = r;
}

}  // namespace

int launch_rotate(const DevIndex& ix, const float* q, int nq, float* out, cudaStream_t s) {
    int td = 1;
    while ((td << 1) <= ix.dim) td <<= 1;
    const float fac = 1.0f / sqrtf(static_cast<float>(td));
    if (!launch_rotate_warp(ix.dim, ix.pd, td, q, nq, fac, ix.signs, ix.mean_rot, out, s))
        rotate_queries_kernel<<<nq, 256, ix.pd * sizeof(float), s>>>(q, ix.dim, ix.pd, td, fac,
                                                                     ix.signs, ix.mean_rot, out);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_rotate_raw(const uint8_t* signs, int dim, int pd, const float* src, int n, float* dst,
                      const float* subtract, cudaStream_t s) {
    int td = 1;
    while ((td << 1) <= dim) td <<= 1;
    const float fac = 1.0f / sqrtf(static_cast<float>(td));
    if (!launch_rotate_warp(dim, pd, td, src, n, fac, signs, subtract, dst, s))
        rotate_queries_kernel<<<n, 256, pd * sizeof(float), s>>>(src, dim, pd, td, fac, signs,
                                                                 subtract, dst);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_route_one(const DevIndex& ix, const float* rq, int nprobe, const RouteWork& w,
                     cudaStream_t s) {
    const int warps = 8;
    int grid = (ix.nlist + warps - 1) / warps;  // one centroid per warp
    grid = grid < 1 ? 1 : (grid > 1184 ? 1184 : grid);
    // dynamic shared memory: the query, reused by the last CTA for the keys
    // (up to 8 * 256 lists: their first tiles and lengths; more: the keys,
    // up to 64 KB of them)
    const size_t lists_bytes = ix.nlist <= static_cast<size_t>(kRegKeys) * warps * 32
                                   ? (2 * static_cast<size_t>(ix.nlist) + 8) * 4
                                   : std::min<size_t>(ix.nlist * 8, 64 * 1024);
    size_t dyn = std::max<size_t>(ix.pd * sizeof(float), lists_bytes);
    if (dyn > 48 * 1024) {
        static size_t configured[64] = {};
        int dev = 0;
        E8QC_CUDA(cudaGetDevice(&dev));
        if (configured[dev & 63] < dyn) {
            E8QC_CUDA(cudaFuncSetAttribute(route_one_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(dyn)));
            configured[dev & 63] = dyn;
        }
    }
    route_one_kernel<<<grid, warps * 32, dyn, s>>>(ix, rq, nprobe, w, static_cast<unsigned>(dyn));
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

// Synthetic rotated queries for tuning runs: row i = 0.75 * c_a + 0.25 * c_b
// for two centroids picked by a hash of (seed, i) -- points near the lists,
// so routing and list loads look like a real batch's.
__global__ void synth_queries_kernel(const float* __restrict__ cen, int nlist, int pd, unsigned long long seed,
                                     float* __restrict__ out) {
    unsigned long long h = seed + 0x9E3779B97F4A7C15ull * (blockIdx.x + 1ull);
    h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
    h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
    h ^= h >> 31;
    const int a = static_cast<int>((h & 0xFFFFFFFFull) % static_cast<unsigned>(nlist));
    const int b = static_cast<int>((h >> 32) % static_cast<unsigned>(nlist));
    for (int i = threadIdx.x; i < pd; i += blockDim.x)
        out[static_cast<size_t>(blockIdx.x) * pd + i] =
            0.75f * cen[static_cast<size_t>(a) * pd + i] + 0.25f * cen[static_cast<size_t>(b) * pd + i];
}

int launch_synth_queries(const DevIndex& ix, int nq, unsigned long long seed, float* out, cudaStream_t s) {
    synth_queries_kernel<<<nq, 256, 0, s>>>(ix.cen, ix.nlist, ix.pd, seed, out);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_probe_bound(const DevIndex& ix, const float* rq, const float* rx, const uint32_t* qsel,
                       const uint32_t* slot_of, const uint32_t* list_of, const double* dlev, const double* mid, int m,
                       int dim, double* out, cudaStream_t s) {
    if (m <= 0) return 0;
    const int grid = (m + 7) / 8;
    switch (ix.bits) {
#define E8QC_CASE(b)                                                                                              \
    case b:                                                                                                       \
        probe_bound_kernel<b><<<grid, 256, 0, s>>>(ix, rq, rx, qsel, slot_of, list_of, dlev, mid, m, dim, out); \
        break;
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_estimate(const DevIndex& ix, const float* rq, int list, uint32_t slot, float* out,
                    cudaStream_t s) {
    switch (ix.bits) {
#define E8QC_CASE(b) \
    case b: estimate_kernel<b><<<1, 32, 0, s>>>(ix, rq, list, slot, out); break;
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

}  // namespace e8qc
