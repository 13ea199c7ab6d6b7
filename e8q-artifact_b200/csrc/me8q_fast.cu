// The reference's production ME8Q search (Me8qIndex::SearchIVFFast*) on the
// device: its fast layout (BuildFastLayout, src/index/me8q_fast.cpp:37-307)
// built from the index's code streams, and a batched form of its cascade
// (ScanPreRouted, me8q_fast.cpp:548-1090; CoarsePruneAvx512,
// src/simd/me8q_prune_avx512.cpp:9-92).
//
// Layout (per 32-slot tile t, as the reference's 32-row batches):
//   plane  [t][colw][32] words: plane column c (8 dims of a coded run) of
//          lane l is byte c%4 of word (t*colw + c/4)*32 + l; its bits are the
//          top bit of each digit (rate 1: the sign bits of dims 0..6 and the
//          branch in bit 0), dim 0 in bit 7;
//   gain, vpc [run][slot]: the zero-parallel-residual fit on the scan basis
//          w = pbar[top bit], as (gain, vpc) with exact undo
//          h2 - 2 coef (vpc + gain S);
//   bank   [t][run][96]: base (floor), weight (nearest), perp (ceil) u8;
//   scl    [t][run][8]: their (min, step) pairs.
//
// Search, per batch of queries (route and per-query select shared with the
// grouped exact scan):
//   me8q_lut_kernel     one CTA per query: the float LUT of every column (16
//                       entries per nibble half), quantised to u8 over its
//                       range as QuantizeLut does, and the per-run scalars;
//   me8q_cascade_kernel one warp per query: the reference's scan in its own
//                       order (probes by (d2, list), 32-row batches, the
//                       filter's lanes, groups of 4, the live heap), so every
//                       prune decision is taken against the same k-th
//                       distance as the reference's. Coarse accumulators and
//                       the fp32 filter run lane-parallel, each run's exact
//                       score is split over the lanes.
// The arithmetic is the reference's, fused multiply-adds where its compiler
// fuses them; the exact run scores sum in another order than its AVX-512
// kernel, so a distance can differ in its last bits.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "device_common.cuh"
#include "me8q.h"
#include "me8q_stream.cuh"

namespace e8qc {

namespace {

constexpr int kFastWarps = 8;  // warps of the pruned scan / seed CTAs

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

// ---- build ------------------------------------------------------------------

// One thread per (slot, coded run): plane bytes and the fit of
// me8q_fast.cpp:140-230 in fp64 (this file builds with --fmad=false: the
// fused multiply-adds are the fma() written here, the ones the reference's
// compiler forms).
__global__ void me8q_fast_fit_kernel(Me8qView v, Me8qFast f, uint8_t* __restrict__ plane_b,
                                     float* __restrict__ gain, float* __restrict__ vpc, float* __restrict__ perp) {
    const size_t gid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t slot = gid / static_cast<size_t>(f.nrun);
    const int r = static_cast<int>(gid - slot * static_cast<size_t>(f.nrun));
    if (slot >= v.nslots) return;
    if (v.base.ids[slot] == 0xFFFFFFFFu) return;
    const Me8qFastRun run = f.runs[r];
    const uint32_t L = v.base.list_of_tile[slot >> 5];
    const float* rc = v.base.cen + static_cast<size_t>(L) * v.base.pd + run.off;
    const float* lev0 = v.levels + run.lev;
    const int q = 1 << run.bits;
    const size_t tile = slot >> 5;
    const int lane = static_cast<int>(slot & 31);
    double dot_ew = 0.0, n2_w = 0.0, n2_e = 0.0, dot_ce = 0.0, dot_cw = 0.0;
    for (int j = 0; j < run.len / 8; ++j) {
        uint32_t dg[8];
        const int br = me8q_block(v.base.codes, v.base.nch, slot, run.word0, run.bits, j, dg);
        const float* lev = lev0 + br * q;
        uint32_t byte = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const uint32_t top = (run.bits == 1 && t == 7) ? static_cast<uint32_t>(br) : (dg[t] >> (run.bits - 1)) & 1u;
            byte |= top << (7 - t);
            const double ve = static_cast<double>(lev[dg[t]]);
            const double wc = (run.bits == 1 && t == 7) ? 0.0 : static_cast<double>(top ? run.p1 : run.p0);
            const double cv = static_cast<double>(rc[j * 8 + t]);
            dot_ew = fma(ve, wc, dot_ew);
            n2_w = fma(wc, wc, n2_w);
            n2_e = fma(ve, ve, n2_e);
            dot_ce = fma(cv, ve, dot_ce);
            dot_cw = fma(cv, wc, dot_cw);
        }
        const int col = run.blk0 + j;
        plane_b[((tile * f.colw + (col >> 2)) * 32 + lane) * 4 + (col & 3)] = static_cast<uint8_t>(byte);
    }
    const size_t o = static_cast<size_t>(r) * v.nslots + slot;
    const double coef = static_cast<double>(v.coef[o]);
    const double h2 = static_cast<double>(v.h2[o]);
    double rn2 = fma(-(2.0 * coef), dot_ce, h2);
    if (rn2 < 0.0) rn2 = 0.0;
    const double rn = sqrt(rn2);
    const double sqrt_lm1 = sqrt(static_cast<double>(run.len - 1 > 1 ? run.len - 1 : 1));
    const double abs_c = fabs(coef);
    float g = 0.0f, vp = 0.0f, pp = 0.0f;
    if (n2_e > 1e-30 && abs_c > 1e-30) {
        const double ve_norm = sqrt(n2_e);
        const double n2_w_safe = n2_w > 1e-30 ? n2_w : 1e-30;
        const double dot_uw = dot_ew / ve_norm;
        const double uw_eps = 1e-12 * sqrt(n2_w_safe);
        double wx, norm_rx;
        if (fabs(dot_uw) > uw_eps) {
            wx = 2.0 * rn / dot_uw;
            const double rx2 = fma(-(4.0 * coef * wx), dot_ew, fma(4.0 * coef * coef, n2_e, wx * wx * n2_w));
            norm_rx = sqrt(rx2 > 0.0 ? rx2 : 0.0);
        } else {
            const double gamma = dot_ew / n2_w_safe;
            wx = 2.0 * coef * gamma;
            double vp2 = fma(-(gamma * gamma), n2_w, n2_e);
            if (vp2 < 0.0) vp2 = 0.0;
            norm_rx = 2.0 * abs_c * sqrt(vp2);
        }
        g = static_cast<float>(wx / (2.0 * abs_c));
        vp = static_cast<float>(fma(-wx, dot_cw, h2 - rn2) / (2.0 * abs_c));
        pp = static_cast<float>((norm_rx / sqrt_lm1) / (2.0 * abs_c));
    } else if (n2_w > 1e-30) {
        const double gamma = dot_ew / n2_w;
        double vp2 = fma(-(gamma * gamma), n2_w, n2_e);
        if (vp2 < 0.0) vp2 = 0.0;
        g = static_cast<float>(gamma);
        vp = static_cast<float>(fma(-gamma, dot_cw, dot_ce));
        pp = static_cast<float>(sqrt(vp2) / sqrt_lm1);
    }
    gain[o] = g;
    vpc[o] = vp;
    perp[o] = pp;
}

// One warp per (tile, run): the u8 banks of me8q_fast.cpp:250-300 over the
// tile's live lanes.
__global__ void me8q_fast_bank_kernel(Me8qView v, Me8qFast f, const float* __restrict__ perp,
                                      uint8_t* __restrict__ bank, float* __restrict__ scl, size_t nwork) {
    const size_t w = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nwork) return;
    const size_t tile = w / static_cast<size_t>(f.nrun);
    const int r = static_cast<int>(w - tile * static_cast<size_t>(f.nrun));
    const size_t slot = tile * 32 + lane;
    const bool live = v.base.ids[slot] != 0xFFFFFFFFu;
    const size_t o = static_cast<size_t>(r) * v.nslots + slot;
    float val[3] = {0.0f, 0.0f, 0.0f};
    if (live) {
        const float coef = v.coef[o], h2 = v.h2[o];
        val[0] = fmaf(-(2.0f * coef), f.vpc[o], h2);
        val[1] = 2.0f * coef * f.gain[o];
        val[2] = perp[o] * 2.0f * fabsf(coef);
    }
    float sc[3], mn[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float lo = live ? val[c] : inf_f(), hi = live ? val[c] : -inf_f();
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(kFull, lo, s));
            hi = fmaxf(hi, __shfl_xor_sync(kFull, hi, s));
        }
        mn[c] = lo;
        sc[c] = hi > lo ? __fdiv_rn(__fsub_rn(hi, lo), 255.0f) : 1.0f;
    }
    uint8_t* bp = bank + w * 96;
    int q0 = 0, q1 = 0, q2 = 0;
    if (live) {
        q0 = static_cast<int>(__fdiv_rn(__fsub_rn(val[0], mn[0]), sc[0]));
        q1 = static_cast<int>(roundf(__fdiv_rn(__fsub_rn(val[1], mn[1]), sc[1])));
        q2 = static_cast<int>(ceilf(__fdiv_rn(__fsub_rn(val[2], mn[2]), sc[2])));
    }
    bp[lane] = static_cast<uint8_t>(min(max(q0, 0), 255));
    bp[32 + lane] = static_cast<uint8_t>(min(max(q1, 0), 255));
    bp[64 + lane] = static_cast<uint8_t>(min(max(q2, 0), 255));
    if (lane < 8) {
        const float out[8] = {mn[0], sc[0], mn[1], sc[1], mn[2], sc[2], 0.0f, 0.0f};
        float o8 = out[0];
#pragma unroll
        for (int i = 1; i < 8; ++i)
            if (lane == i) o8 = out[i];
        scl[w * 8 + lane] = o8;
    }
}

// One thread per (list, run): ||rc_r||^2 in fp64, sequential.
__global__ void me8q_fast_rcn2_kernel(Me8qView v, Me8qFast f, double* __restrict__ rc_n2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.base.nlist * f.nrun) return;
    const int L = i / f.nrun, r = i - L * f.nrun;
    const Me8qFastRun run = f.runs[r];
    const float* rc = v.base.cen + static_cast<size_t>(L) * v.base.pd + run.off;
    double a = 0.0;
    for (int t = 0; t < run.len; ++t) a = fma(static_cast<double>(rc[t]), static_cast<double>(rc[t]), a);
    rc_n2[i] = a;
}

// ---- search -----------------------------------------------------------------

// Per query: LUT floats (smem), range, u8 LUT (global, cols x 32: low
// nibble entries then high nibble entries) and per-run scalars
// qrun[q][r] = {||q_r||^2, lut_min_x, qerr, score_max} (prepare_list,
// me8q_fast.cpp:625-733).
__global__ void me8q_lut_kernel(Me8qFast f, const float* __restrict__ rq, int pd, uint8_t* __restrict__ lut8,
                                double* __restrict__ qrun, float* __restrict__ qdelta) {
    extern __shared__ float lutf[];  // cols * 32
    __shared__ float s_lo[32], s_hi[32];
    const int q = blockIdx.x, tid = threadIdx.x;
    const float* qv = rq + static_cast<size_t>(q) * pd;
    const int n = f.cols * 16;
    float lo = inf_f(), hi = -inf_f();
    for (int e = tid; e < n; e += blockDim.x) {
        const int col = e >> 4, v = e & 15;
        int r = 0;
        while (r + 1 < f.nrun && f.runs[r + 1].blk0 <= col) ++r;
        const Me8qFastRun run = f.runs[r];
        const float* qb = qv + run.off + (col - run.blk0) * 8;
        const float p0 = run.p0, p1 = run.p1;
        const float p70 = run.bits == 1 ? 0.0f : p0, p71 = run.bits == 1 ? 0.0f : p1;
        float a = __fmul_rn(qb[4], ((v >> 3) & 1) ? p1 : p0);
        a = fmaf(qb[5], ((v >> 2) & 1) ? p1 : p0, a);
        a = fmaf(qb[6], ((v >> 1) & 1) ? p1 : p0, a);
        a = fmaf(qb[7], (v & 1) ? p71 : p70, a);
        float b = __fmul_rn(qb[0], ((v >> 3) & 1) ? p1 : p0);
        b = fmaf(qb[1], ((v >> 2) & 1) ? p1 : p0, b);
        b = fmaf(qb[2], ((v >> 1) & 1) ? p1 : p0, b);
        b = fmaf(qb[3], (v & 1) ? p1 : p0, b);
        lutf[col * 32 + v] = a;
        lutf[col * 32 + 16 + v] = b;
        lo = fminf(lo, fminf(a, b));
        hi = fmaxf(hi, fmaxf(a, b));
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(kFull, lo, s));
        hi = fmaxf(hi, __shfl_xor_sync(kFull, hi, s));
    }
    if ((tid & 31) == 0) {
        s_lo[tid >> 5] = lo;
        s_hi[tid >> 5] = hi;
    }
    __syncthreads();
    lo = s_lo[0];
    hi = s_hi[0];
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) {
        lo = fminf(lo, s_lo[w]);
        hi = fmaxf(hi, s_hi[w]);
    }
    const float delta = hi > lo ? __fdiv_rn(__fsub_rn(hi, lo), 255.0f) : 1.0f;
    uint8_t* out = lut8 + static_cast<size_t>(q) * f.cols * 32;
    for (int e = tid; e < f.cols * 32; e += blockDim.x) {
        const int vq = static_cast<int>(__fadd_rn(__fdiv_rn(__fsub_rn(lutf[e], lo), delta), 0.5f));
        out[e] = static_cast<uint8_t>(min(max(vq, 0), 255));
    }
    if (tid < f.nrun) {
        const Me8qFastRun run = f.runs[tid];
        double a = 0.0;
        for (int t = 0; t < run.len; ++t)
            a = fma(static_cast<double>(qv[run.off + t]), static_cast<double>(qv[run.off + t]), a);
        const int nblk = run.len / 8;
        const double lmx = static_cast<double>(lo) * (2.0 * nblk);
        const float sq = static_cast<float>(sqrt(static_cast<double>(nblk > 1 ? nblk : 1)));
        const double qerr = static_cast<double>(__fmul_rn(__fmul_rn(2.0f, sq), delta));
        const double top = fma(2.0 * nblk * 255.0, static_cast<double>(delta), lmx);
        double* o = qrun + (static_cast<size_t>(q) * f.nrun + tid) * 4;
        o[0] = a;
        o[1] = lmx;
        o[2] = qerr;
        o[3] = fabs(lmx) > fabs(top) ? fabs(lmx) : fabs(top);
    }
    if (tid == 0) qdelta[q] = delta;
}

// The exact fp32 score of one coded run of one slot (ScoreRunSplit*,
// src/simd/me8q_score_generic.cpp:100-126): sum over the run's dims of
// q * level, a chain per block, the lanes splitting the blocks; returns the
// warp total.
__device__ __forceinline__ float run_score_warp(const uint4* codes, int nch, const float* levels,
                                                const Me8qFastRun& run, size_t slot, const float* qv) {
    const int lane = threadIdx.x & 31;
    const float* lev0 = levels + run.lev;
    float acc = 0.0f;
    for (int j = lane; j < run.len / 8; j += 32) {
        uint32_t dg[8];
        const int br = me8q_block(codes, nch, slot, run.word0, run.bits, j, dg);
        const float* lev = lev0 + br * (1 << run.bits);
        const float* qb = qv + run.off + j * 8;
        float b = 0.0f;
#pragma unroll
        for (int t = 0; t < 8; ++t) b = fmaf(qb[t], __ldg(lev + dg[t]), b);
        acc = __fadd_rn(acc, b);
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(kFull, acc, s));
    return acc;
}

// The reference's heap (PushCandidate, src/index/me8q_search.cpp:121-134):
// ascending distance, a new row before the rows of equal distance, nothing
// enters a full heap unless strictly below its last distance. Entry j of
// the k <= 128 lives in slot j / 32 of lane j % 32; all members are called
// by the whole warp with uniform arguments.
struct WarpHeap {
    float d[4];
    uint32_t id[4];
    int cnt, k;

    __device__ void init(int k_) {
        k = k_;
        cnt = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            d[s] = inf_f();
            id[s] = 0xFFFFFFFFu;
        }
    }
    __device__ __forceinline__ float back() const {
        const int j = cnt - 1, s = j >> 5;
        float x = d[0];
        if (s == 1) x = d[1];
        if (s == 2) x = d[2];
        if (s == 3) x = d[3];
        return __shfl_sync(kFull, x, j & 31);
    }
    // the heap's k-th distance, +inf while it holds fewer than k rows
    __device__ __forceinline__ float distk() const { return cnt < k ? inf_f() : back(); }
    __device__ void push(float dist, uint32_t pid) {
        if (cnt >= k && !(dist < back())) return;
        const int lane = threadIdx.x & 31;
        int pos = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) pos += __popc(__ballot_sync(kFull, s * 32 + lane < cnt && d[s] < dist));
#pragma unroll
        for (int s = 3; s >= 0; --s) {
            float pd = __shfl_up_sync(kFull, d[s], 1);
            uint32_t pi = __shfl_up_sync(kFull, id[s], 1);
            if (s > 0) {
                const float cd2 = __shfl_sync(kFull, d[s > 0 ? s - 1 : 0], 31);
                const uint32_t ci2 = __shfl_sync(kFull, id[s > 0 ? s - 1 : 0], 31);
                if (lane == 0) {
                    pd = cd2;
                    pi = ci2;
                }
            }
            const int j = s * 32 + lane;
            if (j > pos) {
                d[s] = pd;
                id[s] = pi;
            } else if (j == pos) {
                d[s] = dist;
                id[s] = pid;
            }
        }
        if (cnt < k) ++cnt;
    }
};

// Per-warp shared memory of the cascade kernel (sizes in bytes).
// The u8 LUT first (16-byte aligned), then fp64 sqrt(d2_r), the query's
// per-run scalars and the group's
// s_c and t (4 members), the group's (coef, h2, gain, vpc) per (member,
// run), then acc, s_c and t per (run, lane), then two tile
// stages (the tile's plane words, then per run its 96 bank bytes and 8
// scales); a multiple of 16 bytes so every warp's slice stays aligned.
__host__ __device__ inline size_t cascade_stage_words(int cols, int nrun) {
    return static_cast<size_t>((cols + 3) / 4) * 32 + static_cast<size_t>(nrun) * 32;
}
__host__ __device__ inline size_t cascade_warp_bytes(int cols, int nrun) {
    const size_t b = static_cast<size_t>(cols) * 32 + static_cast<size_t>(nrun) * 8 * (1 + 4 + 8) +
                     static_cast<size_t>(nrun) * 4 * 4 * 4 + 128 + static_cast<size_t>(nrun) * 32 * 4 * 3 +
                     2 * cascade_stage_words(cols, nrun) * 4;
    return (b + 15) / 16 * 16;
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Stage tile `tile` (plane words, banks and scales) into one of the warp's
// two buffers, asynchronously (one commit group per tile).
__device__ __forceinline__ void stage_tile(const Me8qFast& f, size_t tile, uint32_t* dst) {
    const int lane = threadIdx.x & 31;
    const uint32_t* src = f.plane + tile * f.colw * 32;
    for (int w = 0; w < f.colw; ++w) cp_async4(dst + w * 32 + lane, src + w * 32 + lane);
    uint32_t* bd = dst + f.colw * 32;
    for (int r = 0; r < f.nrun; ++r) {
        const uint32_t* bs = lane < 24 ? reinterpret_cast<const uint32_t*>(f.bank + (tile * f.nrun + r) * 96) + lane
                                       : reinterpret_cast<const uint32_t*>(f.scl + (tile * f.nrun + r) * 8) + (lane - 24);
        cp_async4(bd + r * 32 + lane, bs);
    }
    cp_async_commit();
}

// flush4 (me8q_fast.cpp:830-960) for a group of bn <= 4 members: the runs
// in the order of the group's mean t^2 per block (largest first, ties in
// run order), each run's exact score replacing its coarse term, death once
// the remaining slack cannot bring a member under dk. Writes the members'
// distances to dist and returns the mask of the dead. Out of line: one copy
// of this rarely-run code keeps the scan loop's instruction stream small.
struct FlushArgs {
    const uint4* codes;
    const float *coef, *h2, *gain, *vpc, *levels;
    const Me8qFastRun* runs;  // the CTA's shared copy
    size_t nslots;
    int nch, nr;
};

static __device__ __noinline__ unsigned flush_group(const FlushArgs fa, const float* qv, size_t tile, int bn, double d2,
                                                    float lambda, double dk, const int* g_ln, const double* g_pq,
                                                    const double* g_sc, const double* g_tr, float* g_fac,
                                                    double* dist) {
    const int lane = threadIdx.x & 31;
    const int nr = fa.nr;
    // the group's factors, one load per (member, run)
    for (int i = lane; i < bn * nr; i += 32) {
        const int j = i / nr, r = i - j * nr;
        const size_t o = static_cast<size_t>(r) * fa.nslots + tile * 32 + g_ln[j];
        float* fo = g_fac + (j * nr + r) * 4;
        fo[0] = __ldg(fa.coef + o);
        fo[1] = __ldg(fa.h2 + o);
        fo[2] = __ldg(fa.gain + o);
        fo[3] = __ldg(fa.vpc + o);
    }
    __syncwarp();
    int order[kFastMaxRuns];
    double mean[kFastMaxRuns];
    for (int r = 0; r < nr; ++r) {
        order[r] = r;
        double a = 0.0;
        for (int j = 0; j < bn; ++j) a = fma(g_tr[j * nr + r], g_tr[j * nr + r], a);
        const int nb = fa.runs[r].len / 8;
        mean[r] = __ddiv_rn(a, static_cast<double>(nb > 1 ? nb : 1));
    }
    for (int a = 1; a < nr; ++a)
        for (int z = a; z > 0 && mean[order[z]] > mean[order[z - 1]]; --z) {
            const int t = order[z];
            order[z] = order[z - 1];
            order[z - 1] = t;
        }
    double dj[4], rem[4];
    unsigned dead = 0;
    for (int j = 0; j < 4; ++j) {
        rem[j] = j < bn ? g_pq[2 * j] : 0.0;
        dj[j] = d2;
        if (j >= bn) {
            dead |= 1u << j;
            continue;
        }
        if (nr == 1) {
            dj[j] = __dadd_rn(d2, static_cast<double>(g_fac[j * 4 + 1]));
        } else {
            double dcc = d2;
            for (int r = 0; r < nr; ++r) {
                const float* fo = g_fac + (j * nr + r) * 4;
                dcc = __dadd_rn(dcc, fma(-(2.0 * static_cast<double>(fo[0])),
                                         fma(static_cast<double>(fo[2]), g_sc[j * nr + r], static_cast<double>(fo[3])),
                                         static_cast<double>(fo[1])));
            }
            dj[j] = dcc;
        }
    }
    for (int oi = 0; oi < nr; ++oi) {
        const int r = order[oi];
        const Me8qFastRun run = fa.runs[r];
#pragma unroll 1
        for (int j = 0; j < bn; ++j) {
            if ((dead >> j) & 1u) continue;
            const float* fo = g_fac + (j * nr + r) * 4;
            const double coef = static_cast<double>(fo[0]);
            const double s_ex = static_cast<double>(run_score_warp(fa.codes, fa.nch, fa.levels, run, tile * 32 + g_ln[j], qv));
            if (nr == 1) {
                dj[j] = fma(-(2.0 * coef), s_ex, dj[j]);
            } else {
                const double u = fma(static_cast<double>(fo[2]), g_sc[j * nr + r], static_cast<double>(fo[3]));
                dj[j] = fma(2.0 * coef, __dsub_rn(u, s_ex), dj[j]);
            }
            const double t = g_tr[j * nr + r];
            rem[j] = fma(-t, t, rem[j]);
            if (__dsub_rn(fma(-static_cast<double>(lambda), sqrt(rem[j] > 0.0 ? rem[j] : 0.0), dj[j]),
                          g_pq[2 * j + 1]) >= dk)
                dead |= 1u << j;
        }
    }
    if (lane == 0)
        for (int j = 0; j < bn; ++j) dist[j] = dj[j];
    __syncwarp();
    return dead;
}

// One warp per query: the reference's ScanPreRouted (me8q_fast.cpp:548-1090)
// in its own order -- probes by (d2, list), batches of 32 rows, the fp32
// filter of CoarsePruneAvx512 on the first 16*floor(m/16) lanes against the
// heap's k-th distance at the batch start, then each kept lane in order
// against the live heap (the filter's values, or the fp64 scalar twin on
// the tail lanes), groups of 4 through the run cascade (flush4) and into the
// heap. Coarse accumulators and the filter run lane-parallel, run scores
// warp-cooperatively; everything else is warp-uniform.
__global__ void __launch_bounds__(kFastWarps * 32, 2) me8q_cascade_kernel(
    Me8qView v, Me8qFast f, const float* __restrict__ rq, const uint8_t* __restrict__ lut8,
    const double* __restrict__ qrun, const float* __restrict__ qdelta, const uint32_t* __restrict__ probes,
    const float* __restrict__ pd2, int nq, int np, int k, float lambda, int out_stride, uint32_t* __restrict__ out_ids,
    float* __restrict__ out_d, unsigned long long* __restrict__ counts) {
    extern __shared__ __align__(16) uint8_t fsm[];
    __shared__ Me8qFastRun s_runs[kFastMaxRuns];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < f.nrun) s_runs[threadIdx.x] = f.runs[threadIdx.x];
    __syncthreads();
    const int q = blockIdx.x * kFastWarps + warp;
    if (q >= nq) return;  // warp-uniform; no block barrier follows
    const int nr = f.nrun, cols = f.cols;
    const FlushArgs fa{v.base.codes, v.coef, v.h2, f.gain, f.vpc, v.levels, s_runs, v.nslots, v.base.nch, nr};
    uint8_t* base = fsm + static_cast<size_t>(warp) * cascade_warp_bytes(cols, nr);
    const int lut_bytes = cols * 32;
    uint8_t* lut = base;                                             // cols x 32
    double* s_sd2 = reinterpret_cast<double*>(base + lut_bytes);     // nr
    double* s_qr = s_sd2 + nr;                                       // nr x {qn2, lut_min_x, qerr, score_max}
    double* g_sc = s_qr + 4 * nr;                                    // 4 x nr
    double* g_tr = g_sc + 4 * nr;                                    // 4 x nr
    double* g_pq = g_tr + 4 * nr;                                    // 4 x (pool, qadd)
    double* g_dist = g_pq + 8;                                       // 4 flushed distances
    int* g_ln = reinterpret_cast<int*>(g_dist + 4);                  // 4 member lanes (+ pad)
    float* g_fac = reinterpret_cast<float*>(g_ln + 8);               // 4 x nr x 4
    int* s_acc = reinterpret_cast<int*>(g_fac + 16 * nr);            // nr x 32
    float* s_sc = reinterpret_cast<float*>(s_acc + nr * 32);         // nr x 32
    float* s_tr = s_sc + nr * 32;                                    // nr x 32
    uint32_t* stg = reinterpret_cast<uint32_t*>(s_tr + nr * 32);     // 2 tile stages
    const int stg_words = static_cast<int>(cascade_stage_words(cols, nr));
    {
        const uint4* src = reinterpret_cast<const uint4*>(lut8 + static_cast<size_t>(q) * lut_bytes);
        uint4* dst = reinterpret_cast<uint4*>(lut);
        for (int e = lane; e < lut_bytes / 16; e += 32) dst[e] = src[e];
    }
    __syncwarp();
    const float* qv = rq + static_cast<size_t>(q) * v.base.pd;
    for (int i = lane; i < 4 * nr; i += 32) s_qr[i] = qrun[static_cast<size_t>(q) * nr * 4 + i];
    __syncwarp();
    const double* qr0 = s_qr;  // per run {qn2, lut_min_x, qerr, score_max}
    const float delta = qdelta[q];
    const uint32_t* pr = probes + static_cast<size_t>(q) * np;
    const float* pdq = pd2 + static_cast<size_t>(q) * np;
    WarpHeap heap;
    heap.init(k);
    unsigned long long n_cand = 0, n_surv = 0;
    unsigned long long last = 0;
    for (int it = 0; it < np; ++it) {
        // the next probe in (d2 bits, list id) order (RouteQuery's order)
        unsigned long long best = ~0ull;
        for (int p = lane; p < np; p += 32) {
            const unsigned long long key = (static_cast<unsigned long long>(__float_as_uint(pdq[p])) << 32) | pr[p];
            if ((it == 0 || key > last) && key < best) best = key;
        }
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const unsigned long long o = __shfl_xor_sync(kFull, best, s);
            if (o < best) best = o;
        }
        if (best == ~0ull) break;
        last = best;
        const uint32_t L = static_cast<uint32_t>(best & 0xFFFFFFFFull);
        const float d2f = __uint_as_float(static_cast<uint32_t>(best >> 32));
        const double d2 = static_cast<double>(d2f);
        const uint32_t len = v.base.list_len[L], tile0 = v.base.tile_begin[L];
        if (len == 0) continue;
        // sqrt(d2_r) per run (fp64; the dot split over the lanes)
        for (int r = 0; r < nr; ++r) {
            const Me8qFastRun run = s_runs[r];
            const float* rc = v.base.cen + static_cast<size_t>(L) * v.base.pd + run.off;
            double dot = 0.0;
            for (int t = lane; t < run.len; t += 32)
                dot = fma(static_cast<double>(qv[run.off + t]), static_cast<double>(rc[t]), dot);
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) dot = __dadd_rn(dot, __shfl_xor_sync(kFull, dot, s));
            const double d2r = fma(-2.0, dot, __dadd_rn(qr0[r * 4], f.rc_n2[static_cast<size_t>(L) * nr + r]));
            if (lane == 0) s_sd2[r] = sqrt(d2r > 0.0 ? d2r : 0.0);
        }
        __syncwarp();
        stage_tile(f, tile0, stg);
        for (uint32_t i0 = 0; i0 < len; i0 += 32) {
            const int m = static_cast<int>(min(32u, len - i0));
            const size_t tile = tile0 + (i0 >> 5);
            const int covered = m >= 16 ? (m / 16) * 16 : 0;
            const float distk0 = heap.distk();
            const float sdk = distk0 < inf_f() ? sqrtf(fmaxf(distk0, 0.0f)) : inf_f();
            // the next tile streams in while this one is scored
            const int buf = static_cast<int>((i0 >> 5) & 1u);
            if (i0 + 32 < len) {
                stage_tile(f, tile + 1, stg + (buf ^ 1) * stg_words);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            const uint32_t* stp = stg + buf * stg_words;
            const uint8_t* stb = reinterpret_cast<const uint8_t*>(stp + f.colw * 32);  // per run 128 B
            // coarse accumulators (AccumulateCoarseHi) and the fp32 filter
            const uint32_t* pw = stp + lane;
            float dc = d2f, pool = 0.0f, qa = 0.0f, wpad = 0.0f;
            for (int r = 0; r < nr; ++r) {
                const Me8qFastRun run = s_runs[r];
                // a run covers whole plane words (its length is a multiple
                // of 64 dims): one word = 4 columns = 8 LUT entries
                int acc = 0;
#pragma unroll 4
                for (int w = run.blk0 >> 2; w < (run.blk0 + run.len / 8) >> 2; ++w) {
                    const uint32_t word = pw[w * 32];
                    const uint8_t* lc = lut + w * 128;
                    acc += lc[word & 15u] + lc[16 + ((word >> 4) & 15u)] + lc[32 + ((word >> 8) & 15u)] +
                           lc[48 + ((word >> 12) & 15u)] + lc[64 + ((word >> 16) & 15u)] +
                           lc[80 + ((word >> 20) & 15u)] + lc[96 + ((word >> 24) & 15u)] + lc[112 + (word >> 28)];
                }
                s_acc[r * 32 + lane] = acc;
                const double* qr = qr0 + r * 4;
                const uint8_t* bp = stb + r * 128;
                const float* sc = reinterpret_cast<const float*>(bp + 96);
                const float sd2 = static_cast<float>(s_sd2[r]);
                const float rh = sdk < sd2 ? sdk : sd2;
                const float wp = static_cast<float>(0.5 * static_cast<double>(sc[3]) * (qr[3] + qr[2]));
                const float s_c = fmaf(static_cast<float>(acc), delta, static_cast<float>(qr[1]));
                const float base_q = fmaf(static_cast<float>(bp[lane]), sc[1], sc[0]);
                const float weight_q = fmaf(static_cast<float>(bp[32 + lane]), sc[3], sc[2]);
                const float perp_q = fmaf(static_cast<float>(bp[64 + lane]), sc[5], sc[4]);
                dc = fmaf(-weight_q, s_c, dc);
                dc = __fadd_rn(dc, base_q);
                const float t = __fmul_rn(perp_q, rh);
                s_sc[r * 32 + lane] = s_c;
                s_tr[r * 32 + lane] = t;
                pool = fmaf(t, t, pool);
                qa = fmaf(fabsf(weight_q), static_cast<float>(qr[2]), qa);
                wpad = __fadd_rn(wpad, wp);
            }
            const float lane_qa = __fadd_rn(qa, wpad);
            const float slack = fmaf(lambda, sqrtf(pool), lane_qa);
            const bool filtered = lane < covered && __fsub_rn(dc, slack) >= distk0;
            const bool cand = lane < m && !filtered;
            // The reference then walks the kept lanes in order, testing each
            // against the heap's k-th distance at its turn; that distance only
            // changes when a group of 4 is flushed, so the test values are
            // taken lane-parallel and re-taken after each flush. A filter
            // lane's value does not depend on the heap.
            const double val_f = lane < covered
                                     ? __dsub_rn(static_cast<double>(dc),
                                                 fma(static_cast<double>(lambda), sqrt(static_cast<double>(pool)),
                                                     static_cast<double>(lane_qa)))
                                     : 0.0;
            __syncwarp();
            n_cand += static_cast<unsigned long long>(m);
            int bn = 0;
            int pos = -1;  // the last lane taken in order
            for (;;) {
                const float dkf = heap.distk();
                const double distk = static_cast<double>(dkf);
                const double sk = dkf < inf_f() ? sqrt(distk > 0.0 ? distk : 0.0) : static_cast<double>(inf_f());
                // the scalar twin of the tail lanes (me8q_fast.cpp:1000-1040) at this k-th distance
                double val = val_f, t_pool = 0.0, t_qadd = 0.0;
                if (cand && lane >= covered && lane > pos) {
                    double dc_q = d2;
                    for (int r = 0; r < nr; ++r) {
                        const double* qr = qr0 + r * 4;
                        const float* sc = f.scl + (tile * nr + r) * 8;
                        const uint8_t* bp = f.bank + (tile * nr + r) * 96;
                        const double s_cr =
                            fma(static_cast<double>(delta), static_cast<double>(s_acc[r * 32 + lane]), qr[1]);
                        const double base_q = fma(static_cast<double>(bp[lane]), static_cast<double>(sc[1]),
                                                  static_cast<double>(sc[0]));
                        const double weight_q = fma(static_cast<double>(bp[32 + lane]), static_cast<double>(sc[3]),
                                                    static_cast<double>(sc[2]));
                        const double perp_q = fma(static_cast<double>(bp[64 + lane]), static_cast<double>(sc[5]),
                                                  static_cast<double>(sc[4]));
                        dc_q = __dadd_rn(dc_q, fma(-weight_q, s_cr, base_q));
                        const double rh = sk < s_sd2[r] ? sk : s_sd2[r];
                        const double tr = __dmul_rn(perp_q, rh);
                        t_pool = fma(tr, tr, t_pool);
                        t_qadd = fma(fabs(weight_q), qr[2], t_qadd);
                        t_qadd = fma(0.5 * static_cast<double>(sc[3]), __dadd_rn(qr[3], qr[2]), t_qadd);
                    }
                    val = __dsub_rn(dc_q, fma(static_cast<double>(lambda), sqrt(t_pool), t_qadd));
                }
                unsigned pass = __ballot_sync(kFull, cand && lane > pos && !(val >= distk));
                bool full = false;
                while (pass) {
                    const int l = __ffs(pass) - 1;
                    pass &= pass - 1;
                    pos = l;
                    double pool2, qadd;
                    if (l < covered) {
                        pool2 = static_cast<double>(__shfl_sync(kFull, pool, l));
                        qadd = static_cast<double>(__shfl_sync(kFull, lane_qa, l));
                        if (lane < nr) {
                            g_sc[bn * nr + lane] = static_cast<double>(s_sc[lane * 32 + l]);
                            g_tr[bn * nr + lane] = static_cast<double>(s_tr[lane * 32 + l]);
                        }
                    } else {
                        pool2 = __shfl_sync(kFull, t_pool, l);
                        qadd = __shfl_sync(kFull, t_qadd, l);
                        if (lane < nr) {
                            const int r = lane;
                            const double* qr = qr0 + r * 4;
                            const float* sc = f.scl + (tile * nr + r) * 8;
                            const uint8_t* bp = f.bank + (tile * nr + r) * 96;
                            g_sc[bn * nr + r] =
                                fma(static_cast<double>(delta), static_cast<double>(s_acc[r * 32 + l]), qr[1]);
                            const double perp_q = fma(static_cast<double>(bp[64 + l]), static_cast<double>(sc[5]),
                                                      static_cast<double>(sc[4]));
                            g_tr[bn * nr + r] = __dmul_rn(perp_q, sk < s_sd2[r] ? sk : s_sd2[r]);
                        }
                    }
                    if (lane == 0) {
                        g_ln[bn] = l;
                        g_pq[2 * bn] = pool2;
                        g_pq[2 * bn + 1] = qadd;
                    }
                    ++bn;
                    if (bn == 4) {
                        full = true;
                        break;
                    }
                }
                __syncwarp();
                const bool last = !full;  // every passing lane taken: the batch's last group
                if (bn == 0) break;
                const unsigned dmask = flush_group(fa, qv, tile, bn, d2, lambda,
                                                   static_cast<double>(heap.distk()), g_ln, g_pq, g_sc, g_tr, g_fac,
                                                   g_dist);
                for (int j = 0; j < bn; ++j) {
                    if ((dmask >> j) & 1u) continue;
                    ++n_surv;
                    heap.push(static_cast<float>(g_dist[j]), __ldg(v.base.ids + tile * 32 + g_ln[j]));
                }
                bn = 0;
                __syncwarp();
                if (last) break;
            }
        }
    }
    uint32_t* oi = out_ids + static_cast<size_t>(q) * out_stride;
    float* od = out_d + static_cast<size_t>(q) * out_stride;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int j = s * 32 + lane;
        if (j < k) {
            oi[j] = j < heap.cnt ? heap.id[s] : 0xFFFFFFFFu;
            od[j] = j < heap.cnt ? heap.d[s] : inf_f();
        }
    }
    if (lane == 0) {
        atomicAdd(counts, n_cand);
        atomicAdd(counts + 1, n_surv);
    }
}

}  // namespace

int launch_me8q_fast_build(const Me8qView& v, const Me8qFast& f, uint32_t* plane, float* gain, float* vpc,
                           float* perp, uint8_t* bank, float* scl, double* rc_n2, cudaStream_t s) {
    if (f.nrun == 0) return 0;
    const size_t nt = v.nslots * static_cast<size_t>(f.nrun);
    E8QC_CUDA(cudaMemsetAsync(plane, 0, v.nslots / 32 * f.colw * 32 * 4, s));
    Me8qFast fw = f;
    fw.gain = gain;
    fw.vpc = vpc;
    me8q_fast_fit_kernel<<<static_cast<unsigned>((nt + 255) / 256), 256, 0, s>>>(
        v, fw, reinterpret_cast<uint8_t*>(plane), gain, vpc, perp);
    E8QC_CUDA(cudaGetLastError());
    const size_t nwork = v.nslots / 32 * static_cast<size_t>(f.nrun);
    me8q_fast_bank_kernel<<<static_cast<unsigned>((nwork * 32 + 255) / 256), 256, 0, s>>>(v, fw, perp, bank, scl,
                                                                                          nwork);
    E8QC_CUDA(cudaGetLastError());
    const int nrc = v.base.nlist * f.nrun;
    me8q_fast_rcn2_kernel<<<(nrc + 127) / 128, 128, 0, s>>>(v, fw, rc_n2);
    E8QC_CUDA(cudaGetLastError());
    return 3;
}

int me8q_pruned_search(const Me8qView& v, const Me8qFast& f, Workspace& ws, const float* rq, size_t nq, size_t k,
                       size_t nprobe, float lambda, size_t out_stride, uint32_t* out_ids, float* out_d,
                       cudaStream_t s) {
    if (nq == 0) return 0;
    if (f.cols > kFastMaxCols || f.nrun > kFastMaxRuns || f.nrun < 1)
        fail(E8QC_EINVAL, "the ME8Q pruned search supports 1 to 16 coded runs and at most 512 coded blocks");
    const int np = static_cast<int>(nprobe);
    // route + per-query probes (the pair grouping is not used here)
    int launches = batched_prepare(v.base, ws, rq, nq, nullptr, nprobe, 1, 64, 1, s);
    ws.f_lut.ensure(nq * static_cast<size_t>(f.cols) * 32);
    ws.f_qrun.ensure(nq * static_cast<size_t>(f.nrun) * 32);
    ws.f_delta.ensure(nq * 4);
    ws.f_counts.ensure(16);
    E8QC_CUDA(cudaMemsetAsync(ws.f_counts.p, 0, 16, s));
    const size_t lsm = static_cast<size_t>(f.cols) * 32 * 4;
    const size_t csm = static_cast<size_t>(kFastWarps) * cascade_warp_bytes(f.cols, f.nrun);
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    {
        static size_t conf_l[64] = {}, conf_c[64] = {};
        if (lsm > 48 * 1024 && conf_l[dev & 63] < lsm) {
            E8QC_CUDA(cudaFuncSetAttribute(me8q_lut_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(lsm)));
            conf_l[dev & 63] = lsm;
        }
        if (csm > 48 * 1024 && conf_c[dev & 63] < csm) {
            E8QC_CUDA(cudaFuncSetAttribute(me8q_cascade_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(csm)));
            conf_c[dev & 63] = csm;
        }
    }
    me8q_lut_kernel<<<static_cast<unsigned>(nq), 256, lsm, s>>>(f, rq, v.base.pd, ws.f_lut.as<uint8_t>(),
                                                                ws.f_qrun.as<double>(), ws.f_delta.as<float>());
    E8QC_CUDA(cudaGetLastError());
    me8q_cascade_kernel<<<static_cast<unsigned>((nq + kFastWarps - 1) / kFastWarps), kFastWarps * 32, csm, s>>>(
        v, f, rq, ws.f_lut.as<uint8_t>(), ws.f_qrun.as<double>(), ws.f_delta.as<float>(), ws.b_probes.as<uint32_t>(),
        ws.b_pd2.as<float>(), static_cast<int>(nq), np, static_cast<int>(k), lambda, static_cast<int>(out_stride),
        out_ids, out_d, ws.f_counts.as<unsigned long long>());
    E8QC_CUDA(cudaGetLastError());
    return launches + 2;
}

}  // namespace e8qc
