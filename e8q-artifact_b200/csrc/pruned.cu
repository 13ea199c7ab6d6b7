// The reference's production search (E8qIndex::Search with pruning,
// src/index/e8q_search.cpp:215-293; ScanClusterAvx512,
// src/simd/e8q_search_avx512.cpp:552-751) for a batch of queries.
//
// The reference scans lists in probe order with a running k-heap: a coarse
// pass prices one rowA byte per 8-dim block (the digits' top bits) against a
// u8 LUT of the query (PrepareQuery, e8q_search.cpp:20-73), a per-vector
// lower bound from the zero-parallel-residual scan banks (OrthoBatchHeader,
// src/index/e8q_scan_common.hpp:141-156)
//   dlo = (d2 + base - W*S - |W|*lut_err - W_round) - z * r_horizon * Omega
// rejects vectors that cannot beat the heap's current k-th distance, a
// whole-batch test skips 32-row batches, and the survivors are staged 32 at
// a time and refined exactly. Every decision depends on the heap after the
// previous ones, so the GPU gives each query one warp that takes them in the
// reference's order (pruned_cascade_kernel): the 32 rows of a batch are its
// 32 lanes (coarse pass, bound), the staged rows are refined a half-warp per
// row, and the heap is the warp's top-k in the (distance, id) order, the
// reference heap's. pruned_lut_kernel builds the LUTs first (the
// reference's arithmetic: fp64 sums, one u8 step for the table,
// round-to-nearest-even); build_rowa_kernel and ortho_bank_kernel build the
// coarse plane and the scan banks once per index.
#include <cuda_runtime.h>
#include <stdint.h>

#include "decode_accum.cuh"
#include "device_common.cuh"
#include "internal.h"
#include "pruned.h"
#include "scan_common.cuh"
#include "scan_plain.h"

namespace e8qc {

namespace {

using namespace scan1;

// Padded floats per decode unit of the query in shared memory: units are
// whole steps (plus the odd rates' 8-block tail); the 4-float pad puts the
// units that a half-warp's lanes read at once in different banks.
template <int BITS>
__host__ __device__ constexpr int qstep_floats() {
    return ((BITS & 1) ? 16 : 8) * 8 + 4;
}

// Exact score of one vector by a half-warp: lane j of the half decodes units
// j, j + 16, ... of the vector (steps of SBLK blocks, then the tail) and the
// half's lanes sum their partials. `src` = chunk 0 of the vector (chunk c at
// src[c * 32]); `active` false leaves the lane's partial at 0 (the shuffles
// still run: every lane of the warp calls this).
template <int BITS>
__device__ __forceinline__ float exact_half(const uint4* __restrict__ src, bool active, int nsteps, bool tail,
                                            const float* sq, uint32_t tb_addr) {
    using G = StepGeo<BITS>;
    constexpr int SBLK = G::SBLK, SCH = G::SCH, TCH = G::TCH, QS = qstep_floats<BITS>();
    const int j = threadIdx.x & 15;
    float a0 = 0.0f, a1 = 0.0f;
    if (active) {
        for (int u = j; u < nsteps; u += 16) {
            uint4 v[SCH];
            load_chunks(v, src + static_cast<size_t>(u) * SCH * 32);
            accumulate_regs<BITS, SBLK, SCH>(v, reinterpret_cast<const float4*>(sq + u * QS), 0, tb_addr, a0, a1);
        }
        if constexpr ((BITS & 1) != 0) {
            if (tail && (nsteps & 15) == j) {
                uint4 v[TCH];
                load_chunks(v, src + static_cast<size_t>(nsteps) * SCH * 32);
                accumulate_regs<BITS, 8, TCH>(v, reinterpret_cast<const float4*>(sq + nsteps * QS), 0, tb_addr, a0,
                                              a1);
            }
        }
    }
    float S = __fadd_rn(a0, a1);
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) S = __fadd_rn(S, __shfl_xor_sync(kFull, S, o));
    return S;
}

// One tile's coarse pass for this lane's vector: the coarse estimate dc and
// the bound terms P = dc - |W| * lut_err and Omega (perp), from the rowA
// bytes, the tile's bank header and the probe's d2 (the reference's fused
// operations, in its order: src/simd/e8q_search_avx512.cpp:636-676).
struct Coarse {
    float dc, P, perp;
    int acc;  // the u8 LUT sum
};

__device__ __forceinline__ Coarse coarse_lane(const uint4* __restrict__ rowa, int nrc, int B, const uint8_t* lut,
                                              const uint8_t* __restrict__ hdr, float d2, const float* scal) {
    const int lane = threadIdx.x & 31;
    int acc = 0;
    for (int c0 = 0; c0 < nrc; c0 += 8) {
        uint4 v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c0 + c < nrc) v[c] = ld_stream(rowa + static_cast<size_t>(c0 + c) * 32 + lane);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if (c0 + c < nrc) {
                const uint32_t w[4] = {v[c].x, v[c].y, v[c].z, v[c].w};
#pragma unroll
                for (int b = 0; b < 16; ++b) {
                    const int blk = (c0 + c) * 16 + b;
                    if (blk < B) {
                        const uint32_t h = (w[b >> 2] >> ((b & 3) * 8)) & 0xFFu;
                        acc += lut[blk * 32 + (h & 15u)] + lut[blk * 32 + 16 + (h >> 4)];
                    }
                }
            }
        }
    }
    const float* sc = reinterpret_cast<const float*>(hdr + 96);
    const float bmin = __ldg(sc + 0), bsc = __ldg(sc + 1), wmin = __ldg(sc + 2), wsc = __ldg(sc + 3);
    const float pmin = __ldg(sc + 4), psc = __ldg(sc + 5);
    const float bq = static_cast<float>(__ldg(hdr + lane)), wq = static_cast<float>(__ldg(hdr + 32 + lane));
    const float pq = static_cast<float>(__ldg(hdr + 64 + lane));
    const float delta_c = scal[0], base_c = scal[1], lut_err = scal[2], score_max = scal[3];
    const float pad_w_round = __fmul_rn(__fmul_rn(0.5f, wsc), __fadd_rn(score_max, lut_err));
    const float bmin_d2 = __fsub_rn(__fadd_rn(bmin, d2), pad_w_round);
    const float scv = __fmaf_rn(static_cast<float>(acc), delta_c, base_c);
    const float base_term = __fmaf_rn(bq, bsc, bmin_d2);
    const float weight = __fmaf_rn(wq, wsc, wmin);
    Coarse r;
    r.acc = acc;
    r.perp = __fmaf_rn(pq, psc, pmin);
    r.dc = __fmaf_rn(-weight, scv, base_term);
    r.P = __fmaf_rn(-fabsf(weight), lut_err, r.dc);
    return r;
}

// rowA byte of every block of every slot: bit 7 - i = the top bit of stored
// digit field i (digit 7's field holds the branch in its lowest bit, which
// at b = 1 is the whole field: the reference's rowA bit 0 is then the branch).
__global__ void build_rowa_kernel(DevIndex ix, int ntiles, int nrc, uint4* __restrict__ out) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;  // (tile, c, lane)
    const size_t total = static_cast<size_t>(ntiles) * nrc * 32;
    if (i >= total) return;
    const int lane = static_cast<int>(i & 31);
    const size_t tc = i >> 5;
    const int c = static_cast<int>(tc % static_cast<size_t>(nrc));
    const size_t tile = tc / static_cast<size_t>(nrc);
    const uint32_t* base = reinterpret_cast<const uint32_t*>(ix.codes);
    auto word = [&](int w) -> uint32_t {
        // word w of the vector: chunk w/4, component w%4
        const size_t chunk = (tile * ix.nch + static_cast<size_t>(w >> 2)) * 32 + lane;
        return base[chunk * 4 + (w & 3)];
    };
    const int b = ix.bits;
    uint32_t outw[4] = {0u, 0u, 0u, 0u};
    const bool real = ix.ids[tile * 32 + lane] != 0xFFFFFFFFu;
    for (int q = 0; q < 16 && real; ++q) {
        const int blk = c * 16 + q;
        if (blk >= ix.B) break;
        uint32_t byte = 0u;
        for (int d = 0; d < 8; ++d) {
            const long bit = static_cast<long>(blk) * 8 * b + d * b + (b - 1);
            const uint32_t v = (word(static_cast<int>(bit >> 5)) >> (bit & 31)) & 1u;
            byte |= v << (7 - d);
        }
        outw[q >> 2] |= byte << ((q & 3) * 8);
    }
    out[i] = make_uint4(outw[0], outw[1], outw[2], outw[3]);
}

}  // namespace

namespace {

// ---- batched form: one warp per query, the reference's order ---------------

constexpr int kCWarps = 8;  // queries (warps) per CTA of the cascade kernel

// Per query (one CTA): the u8 LUT (B*32 bytes: entry blk*32 + v, v < 16 the
// low nibble, v >= 16 the high one) and its scalars {delta, base, lut_err,
// score_max} (PrepareQuery, src/index/e8q_search.cpp:20-73; the arithmetic of
// the one-query kernel's prologue).
__global__ void pruned_lut_kernel(const float* __restrict__ rq, int pd, int B, int bits, double w0, double w1,
                                  uint8_t* __restrict__ lut8, float* __restrict__ scal) {
    __shared__ unsigned s_hc;
    const int q = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const float* qv = rq + static_cast<size_t>(q) * pd;
    auto cf_of = [&](int e) -> float {
        const int blk = e >> 5, v = e & 15, hi = (e >> 4) & 1;
        const float* qb = qv + blk * 8 + (hi ? 0 : 4);
        double acc = 0.0;
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int bit = (v >> (3 - h)) & 1;
            const int dim = hi ? h : 4 + h;
            const double m = (bits == 1 && dim == 7) ? 0.0 : (bit ? w1 : w0);
            acc = __fma_rn(static_cast<double>(__ldg(qb + h)), m, acc);
        }
        return __double2float_rn(acc);
    };
    if (tid == 0) s_hc = 0u;
    __syncthreads();
    unsigned mx = 0u;
    for (int e = tid; e < B * 32; e += nt) mx = max(mx, __float_as_uint(fabsf(cf_of(e))));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
    if ((tid & 31) == 0) atomicMax(&s_hc, mx);
    __syncthreads();
    const float hc = __uint_as_float(s_hc);
    const float delta = hc > 0.0f ? __fdiv_rn(__fmul_rn(2.0f, hc), 255.0f) : 1.0f;
    const float qinv = __fdiv_rn(1.0f, delta), qoff = __fdiv_rn(hc, delta);
    uint8_t* out = lut8 + static_cast<size_t>(q) * B * 32;
    for (int e = tid; e < B * 32; e += nt) {
        const unsigned u = static_cast<unsigned>(__float2int_rn(__fmaf_rn(cf_of(e), qinv, qoff)));
        out[e] = static_cast<uint8_t>(u > 255u ? 255u : u);
    }
    if (tid == 0) {
        float* sc = scal + static_cast<size_t>(q) * 4;
        sc[0] = delta;
        sc[1] = __fmul_rn(-hc, static_cast<float>(2 * B));
        sc[2] = __fmul_rn(__fmul_rn(2.0f, __fsqrt_rn(static_cast<float>(B))), delta);
        sc[3] = __fmul_rn(static_cast<float>(B), __fmaf_rn(255.0f, delta, __fmul_rn(2.0f, hc)));
    }
}

// Per query (one warp): exclusive prefix over its probes (in the route's list
// order) of their tile counts: toff[qi][p], toff[qi][np] = the query's tiles.
__global__ void pruned_toff_kernel(const DevIndex ix, const uint32_t* __restrict__ probes, int q0, int nqg, int np,
                                   uint32_t* __restrict__ toff) {
    const int lane = threadIdx.x & 31;
    const int qi = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    if (qi >= nqg) return;
    const uint32_t* pr = probes + static_cast<size_t>(q0 + qi) * np;
    uint32_t* out = toff + static_cast<size_t>(qi) * (np + 1);
    uint32_t run = 0;
    for (int p0 = 0; p0 < np; p0 += 32) {
        const int p = p0 + lane;
        const uint32_t t = p < np ? (ix.list_len[pr[p]] + 31u) / 32u : 0u;
        uint32_t inc = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, inc, o);
            if (lane >= o) inc += v;
        }
        if (p < np) out[p] = run + inc - t;
        run += __shfl_sync(kFull, inc, 31);
    }
    if (lane == 0) out[np] = run;
}

// The heap-independent half of every tile a query probes, at full
// parallelism: one warp per (query, tile), lane = row: the u8 LUT sum and the
// bound terms P and Omega (coarse_lane) into [qi][tile][lane] arrays.
__global__ void __launch_bounds__(256) pruned_coarse_kernel(
    const DevIndex ix, const uint8_t* __restrict__ lut8, const float* __restrict__ scal_all,
    const uint32_t* __restrict__ probes, const float* __restrict__ pd2, const uint32_t* __restrict__ toff, int q0,
    int np, size_t max_tiles, PrunedWork pw, int* __restrict__ c_acc, float* __restrict__ c_P,
    float* __restrict__ c_perp) {
    extern __shared__ __align__(16) unsigned char lsm[];
    const int qi = blockIdx.y, q = q0 + qi;
    const int B = ix.B;
    const uint32_t* to = toff + static_cast<size_t>(qi) * (np + 1);
    const uint32_t T = to[np];
    const uint32_t t0 = blockIdx.x * 8u;
    if (t0 >= T) return;  // CTA-uniform, before any barrier
    {
        const uint4* src = reinterpret_cast<const uint4*>(lut8 + static_cast<size_t>(q) * B * 32);
        uint4* dst = reinterpret_cast<uint4*>(lsm);
        for (int e = threadIdx.x; e < B * 2; e += blockDim.x) dst[e] = src[e];
    }
    float scal[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) scal[i] = scal_all[static_cast<size_t>(q) * 4 + i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t t = t0 + (threadIdx.x >> 5);
    if (t >= T) return;
    int lo = 0, hi = np;  // the probe whose tiles hold t: to[lo] <= t < to[lo + 1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (to[mid] <= t) lo = mid;
        else hi = mid;
    }
    const uint32_t L = probes[static_cast<size_t>(q) * np + lo];
    const float d2 = pd2[static_cast<size_t>(q) * np + lo];
    const uint32_t gt = ix.tile_begin[L] + (t - to[lo]);
    const Coarse cr = coarse_lane(pw.rowa + static_cast<size_t>(gt) * pw.nrc * 32, pw.nrc, B, lsm,
                                  pw.banks + static_cast<size_t>(gt) * 128, d2, scal);
    const size_t o = (static_cast<size_t>(qi) * max_tiles + t) * 32 + lane;
    c_acc[o] = cr.acc;
    c_P[o] = cr.P;
    c_perp[o] = cr.perp;
}

// Per-warp shared memory of the cascade kernel: the query in padded units,
// the staged rows (slot, g1, d2 + h3) and their distances.
template <int BITS>
__host__ __device__ inline size_t cascade_warp_bytes(int B) {
    using G = StepGeo<BITS>;
    const int nunits = B / G::SBLK + ((B % G::SBLK) != 0 ? 1 : 0);
    const size_t b = static_cast<size_t>(nunits) * qstep_floats<BITS>() * 4 + 32 * 16;
    return (b + 15) / 16 * 16;
}

// One warp per query: ScanCluster (src/simd/e8q_search_avx512.cpp:552-751)
// over the probes in (d2, list) order with the running heap -- the
// whole-batch skip, the per-lane bound against the heap's k-th distance at
// the batch start, CollectLanes (e8q_scan_common.hpp:86-113: each kept lane
// re-tested against the current k-th, survivors staged, 32 at most, refined
// and inserted when the stage is full and at the end of every list). The
// heap's k-th distance changes only at a flush, so the re-test is a ballot
// taken again after each one. The heap is the warp's top-k in the (distance,
// id) order, the reference heap's order.
template <int BITS>
__global__ void __launch_bounds__(kCWarps * 32, 2) pruned_cascade_kernel(
    DevIndex ix, const float* __restrict__ rq_all, const uint8_t* __restrict__ lut8, const float* __restrict__ scal_all,
    const uint32_t* __restrict__ probes, const float* __restrict__ pd2, int q0, int nqg, int np, int k, PrunedWork pw,
    const uint32_t* __restrict__ toff, size_t max_tiles, const int* __restrict__ c_acc, const float* __restrict__ c_P,
    const float* __restrict__ c_perp, uint32_t* __restrict__ out_ids, float* __restrict__ out_d,
    float* __restrict__ thr_out, unsigned long long* __restrict__ stats) {
    using G = StepGeo<BITS>;
    constexpr int Q = 1 << BITS, REP = table_rep(BITS), SBLK = G::SBLK, QS = qstep_floats<BITS>();
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int B = ix.B;
    const int nsteps = B / SBLK;
    const bool tail = (B % SBLK) != 0;
    const int nunits = nsteps + (tail ? 1 : 0);
    float* tabrep = reinterpret_cast<float*>(smem);  // 2*Q*REP, the CTA's
    for (int e = tid; e < 2 * Q * REP; e += blockDim.x) tabrep[e] = ix.tab[e / REP];
    __syncthreads();
    const int qi = blockIdx.x * kCWarps + warp;
    if (qi >= nqg) return;  // warp-uniform; no block barrier follows
    const int q = q0 + qi;
    const uint32_t* to = toff + static_cast<size_t>(qi) * (np + 1);
    unsigned char* wb = smem + static_cast<size_t>(2 * Q * REP) * 4 +
                        static_cast<size_t>(warp) * cascade_warp_bytes<BITS>(B);
    float* sq = reinterpret_cast<float*>(wb);                                        // nunits*QS
    uint32_t* st_slot = reinterpret_cast<uint32_t*>(sq + nunits * QS);               // 32
    float* st_g1 = reinterpret_cast<float*>(st_slot + 32);                           // 32
    float* st_h3 = st_g1 + 32;                                                       // 32
    float* st_d = st_h3 + 32;                                                        // 32
    const float* rq = rq_all + static_cast<size_t>(q) * ix.pd;
    for (int i = lane; i < ix.pd; i += 32) {
        const int u = i / (SBLK * 8), r = i - u * (SBLK * 8);
        sq[u * QS + r] = rq[i];
    }
    (void)lut8;  // the LUT was applied by pruned_coarse_kernel
    float scal[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) scal[i] = scal_all[static_cast<size_t>(q) * 4 + i];
    __syncwarp();
    const uint32_t tb_addr = smem_addr(tabrep) + static_cast<uint32_t>(lane % REP) * 4u;
    const float lut_err = scal[2], score_max = scal[3], delta_c = scal[0], base_c = scal[1];
    const uint32_t* pr = probes + static_cast<size_t>(q) * np;
    const float* pdq = pd2 + static_cast<size_t>(q) * np;
    WarpTopK top;
    top.init(k);
    int nst = 0;
    unsigned long long n_cand = 0, n_surv = 0;
    // refine the staged rows (a half-warp per row) and insert them
    auto flush = [&]() {
        for (int j0 = 0; j0 < nst; j0 += 2) {
            const int j = j0 + (lane >> 4);
            const bool act = j < nst;
            const uint32_t slot = act ? st_slot[j] : 0u;
            const float S = exact_half<BITS>(ix.codes + static_cast<size_t>(slot >> 5) * ix.nch * 32 + (slot & 31u),
                                             act, nsteps, tail, sq, tb_addr);
            if (act && (lane & 15) == 0) st_d[j] = __fmaf_rn(-__fmul_rn(2.0f, st_g1[j]), S, st_h3[j]);
        }
        __syncwarp();
        const bool in = lane < nst;
        const float dl = in ? st_d[lane] : inf_f();
        top.offer(dl, in, [&] { return __ldg(ix.ids + st_slot[lane]); });
        nst = 0;
        __syncwarp();
    };
    unsigned long long last = 0;
    for (int it = 0; it < np; ++it) {
        unsigned long long best = ~0ull;
        for (int p = lane; p < np; p += 32) {
            const unsigned long long key = (static_cast<unsigned long long>(__float_as_uint(pdq[p])) << 32) | pr[p];
            if ((it == 0 || key > last) && key < best) best = key;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long v = __shfl_xor_sync(kFull, best, o);
            if (v < best) best = v;
        }
        if (best == ~0ull) break;
        last = best;
        const uint32_t L = static_cast<uint32_t>(best & 0xFFFFFFFFull);
        const float d2 = __uint_as_float(static_cast<uint32_t>(best >> 32));
        const uint32_t len = ix.list_len[L], tile0 = ix.tile_begin[L];
        if (len == 0) continue;
        // this probe's position in the route's list order: its tiles' offset
        int pp = 0;
        {
            unsigned found = 0u;
            for (int p0 = 0; p0 < np && found == 0u; p0 += 32) {
                found = __ballot_sync(kFull, p0 + lane < np && pr[p0 + lane] == L);
                if (found) pp = p0 + __ffs(found) - 1;
            }
        }
        const uint32_t tb0 = to[pp];
        const float sqrt_d2 = __fsqrt_rn(d2 > 0.0f ? d2 : 0.0f);
        const size_t cbase = (static_cast<size_t>(qi) * max_tiles + tb0) * 32 + lane;
        int nx_acc = c_acc[cbase];
        float nx_P = c_P[cbase], nx_perp = c_perp[cbase];
        for (uint32_t i0 = 0; i0 < len; i0 += 32) {
            const uint32_t n_logic = min(32u, len - i0);
            const uint32_t gt = tile0 + (i0 >> 5);
            const uint8_t* hdr = pw.banks + static_cast<size_t>(gt) * 128;
            Coarse cr;
            cr.acc = nx_acc;
            cr.P = nx_P;
            cr.perp = nx_perp;
            if (i0 + 32 < len) {  // the next tile's values stream in while this one is decided
                const size_t o = cbase + static_cast<size_t>((i0 >> 5) + 1) * 32;
                nx_acc = c_acc[o];
                nx_P = c_P[o];
                nx_perp = c_perp[o];
            }
            n_cand += n_logic;
            const float distk0 = top.thr_d;
            const float r_h = distk0 < d2 ? __fsqrt_rn(distk0 > 0.0f ? distk0 : 0.0f) : sqrt_d2;
            const float slack = __fmul_rn(pw.z, r_h);
            if (!pw.disable_prune && distk0 < inf_f()) {
                // the whole-batch skip (e8q_search_avx512.cpp:611-635): padding
                // lanes price the zero rowA bytes, as the reference's do
                const float* sc = reinterpret_cast<const float*>(hdr + 96);
                const float bmin = __ldg(sc + 0), wsc = __ldg(sc + 3), pmin = __ldg(sc + 4), psc = __ldg(sc + 5);
                const float wamax = __ldg(sc + 6);
                const float pad_w_round = __fmul_rn(__fmul_rn(0.5f, wsc), __fadd_rn(score_max, lut_err));
                const float pad_add = __fmaf_rn(wamax, lut_err, pad_w_round);
                const float perp_amax = __fmaf_rn(255.0f, psc, pmin);
                int mxa = cr.acc, mna = cr.acc;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    mxa = max(mxa, __shfl_xor_sync(kFull, mxa, o));
                    mna = min(mna, __shfl_xor_sync(kFull, mna, o));
                }
                const float s_hi = __fmaf_rn(static_cast<float>(mxa), delta_c, base_c);
                const float s_lo = __fmaf_rn(static_cast<float>(mna), delta_c, base_c);
                const float s_absmax = fabsf(s_hi) > fabsf(s_lo) ? fabsf(s_hi) : fabsf(s_lo);
                const float lb = __fmaf_rn(-slack, perp_amax,
                                           __fmaf_rn(-wamax, s_absmax, __fsub_rn(__fadd_rn(d2, bmin), pad_add)));
                if (lb >= distk0) continue;
            }
            const float dlo = __fmaf_rn(-slack, cr.perp, cr.P);
            const bool inm = static_cast<uint32_t>(lane) < n_logic && (pw.disable_prune || dlo < distk0);
            int pos = -1;
            for (;;) {
                const float limit = top.thr_d;
                const unsigned pass =
                    __ballot_sync(kFull, inm && lane > pos && (pw.disable_prune || dlo < limit));
                if (pass == 0u) break;
                const int l = __ffs(pass) - 1;
                if (nst == 32) flush();
                if (lane == 0) {
                    const size_t slot = static_cast<size_t>(gt) * 32 + l;
                    st_slot[nst] = static_cast<uint32_t>(slot);
                    st_g1[nst] = __ldg(ix.g1 + slot);
                    st_h3[nst] = __fadd_rn(d2, __ldg(ix.h3 + slot));
                }
                ++nst;
                ++n_surv;
                pos = l;
                __syncwarp();
            }
        }
        if (nst > 0) flush();
    }
    top.store(out_d + static_cast<size_t>(q) * k, out_ids + static_cast<size_t>(q) * k, k);
    if (lane == 0) {
        if (thr_out) thr_out[q] = top.thr_d;
        atomicAdd(stats, n_cand);
        atomicAdd(stats + 1, n_surv);
    }
}

}  // namespace

int launch_pruned_batch(const DevIndex& ix, const float* rq, const uint32_t* probes, const float* pd2, int nq, int np,
                        int k, const PrunedWork& pw, const PrunedScratch& sc, cudaStream_t s) {
    if (nq == 0) return 0;
    int launches = 0;
    pruned_lut_kernel<<<static_cast<unsigned>(nq), 256, 0, s>>>(rq, ix.pd, ix.B, ix.bits, pw.w_cls0, pw.w_cls1,
                                                               sc.lut8, sc.scal);
    E8QC_CUDA(cudaGetLastError());
    ++launches;
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    const void* fn = nullptr;
    size_t smem = 0;
    switch (ix.bits) {
#define E8QC_CASE(b)                                                                                         \
    case b:                                                                                                  \
        fn = reinterpret_cast<const void*>(pruned_cascade_kernel<b>);                                        \
        smem = static_cast<size_t>(2 * (1 << b) * table_rep(b)) * 4 + kCWarps * cascade_warp_bytes<b>(ix.B); \
        break;
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    if (smem > 227 * 1024) fail(E8QC_EINVAL, "the pruned search does not fit this device (padded_dim too large)");
    const size_t lsm = static_cast<size_t>(ix.B) * 32;
    {
        static size_t configured[64][14] = {};
        if (configured[dev & 63][ix.bits] < smem) {
            E8QC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
            configured[dev & 63][ix.bits] = smem;
        }
        static size_t conf_l[64] = {};
        if (lsm > 48 * 1024 && conf_l[dev & 63] < lsm) {
            E8QC_CUDA(cudaFuncSetAttribute(pruned_coarse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(lsm)));
            conf_l[dev & 63] = lsm;
        }
    }
    for (int q0 = 0; q0 < nq; q0 += sc.group) {
        const int g = nq - q0 < sc.group ? nq - q0 : sc.group;
        pruned_toff_kernel<<<static_cast<unsigned>((g + 7) / 8), 256, 0, s>>>(ix, probes, q0, g, np, sc.toff);
        E8QC_CUDA(cudaGetLastError());
        dim3 cg(static_cast<unsigned>((sc.max_tiles + 7) / 8), static_cast<unsigned>(g));
        pruned_coarse_kernel<<<cg, 256, lsm, s>>>(ix, sc.lut8, sc.scal, probes, pd2, sc.toff, q0, np, sc.max_tiles, pw,
                                                  sc.c_acc, sc.c_P, sc.c_perp);
        E8QC_CUDA(cudaGetLastError());
        const unsigned grid = static_cast<unsigned>((g + kCWarps - 1) / kCWarps);
        switch (ix.bits) {
#define E8QC_CASE(b)                                                                                        \
    case b:                                                                                                 \
        pruned_cascade_kernel<b><<<grid, kCWarps * 32, smem, s>>>(ix, rq, sc.lut8, sc.scal, probes, pd2, q0, g, np, k, \
                                                                  pw, sc.toff, sc.max_tiles, sc.c_acc, sc.c_P,   \
                                                                  sc.c_perp, sc.out_ids, sc.out_d, pw.thr, pw.stats); \
        break;
            E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
            E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
            E8QC_CASE(13)
#undef E8QC_CASE
            default: break;
        }
        E8QC_CUDA(cudaGetLastError());
        launches += 3;
    }
    return launches;
}

namespace {

// WriteOrthoBanks (src/index/e8q_build.cpp:33-80) per tile, one warp: the
// live lanes' (base, weight, perp) quantised to u8 over their range (base
// floor, weight nearest, perp ceil) and the 128-byte header: three banks of
// 32 bytes, then min and step of each and max |weight|.
__global__ void ortho_bank_kernel(const float* __restrict__ ortho, const uint32_t* __restrict__ ids, int ntiles,
                                  uint8_t* __restrict__ hdr) {
    const int w = static_cast<int>((static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= ntiles) return;
    const size_t slot = static_cast<size_t>(w) * 32 + lane;
    const bool live = ids[slot] != 0xFFFFFFFFu;
    float val[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) val[c] = live ? ortho[slot * 3 + c] : 0.0f;
    float mn[3], sc[3], mx[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float lo = live ? val[c] : __int_as_float(0x7f800000), hi = live ? val[c] : __int_as_float(0xff800000);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
        }
        mn[c] = lo;
        mx[c] = hi;
        sc[c] = hi > lo ? __fdiv_rn(__fsub_rn(hi, lo), 255.0f) : 1.0f;
    }
    uint8_t* h = hdr + static_cast<size_t>(w) * 128;
    int q0 = 0, q1 = 0, q2 = 0;
    if (live) {
        q0 = static_cast<int>(__fdiv_rn(__fsub_rn(val[0], mn[0]), sc[0]));
        q1 = static_cast<int>(roundf(__fdiv_rn(__fsub_rn(val[1], mn[1]), sc[1])));
        q2 = static_cast<int>(ceilf(__fdiv_rn(__fsub_rn(val[2], mn[2]), sc[2])));
    }
    h[lane] = static_cast<uint8_t>(min(max(q0, 0), 255));
    h[32 + lane] = static_cast<uint8_t>(min(max(q1, 0), 255));
    h[64 + lane] = static_cast<uint8_t>(min(max(q2, 0), 255));
    // scales: bmin, bstep, wmin, wstep, pmin, pstep, max |w|, then zero
    const float out[8] = {mn[0], sc[0], mn[1], sc[1], mn[2], sc[2], fmaxf(fabsf(mn[1]), fabsf(mx[1])), 0.0f};
    float o8 = out[0];
#pragma unroll
    for (int i = 1; i < 8; ++i)
        if (lane == i) o8 = out[i];
    if (lane < 8) reinterpret_cast<float*>(h + 96)[lane] = o8;
}

}  // namespace

int launch_ortho_banks(const float* ortho, const uint32_t* ids, int ntiles, uint8_t* hdr, cudaStream_t s) {
    if (ntiles == 0) return 0;
    ortho_bank_kernel<<<static_cast<unsigned>((static_cast<size_t>(ntiles) * 32 + 255) / 256), 256, 0, s>>>(
        ortho, ids, ntiles, hdr);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_build_rowa(const DevIndex& ix, int ntiles, uint4* rowa, cudaStream_t s) {
    const int nrc = rowa_chunks(ix.B);
    const size_t total = static_cast<size_t>(ntiles) * nrc * 32;
    if (total == 0) return 0;
    build_rowa_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(ix, ntiles, nrc, rowa);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

}  // namespace e8qc
