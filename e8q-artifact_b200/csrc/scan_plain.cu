// Plain one-query streaming scan (the drop-in search path).
//
// Every vector of every probed list gets the exact estimator
//   dist = (d2 + h3) - 2*g1*S,   S = sum_i q[i] * level[branch][digit_i] / sqrt(D)
// (src/simd/e8q_search_generic.cpp:58-66 with d2 folded as at :189) and enters
// a warp top-k; each CTA reduces its warps' lists to one, and the last CTA to
// finish reduces the per-CTA lists to the answer.
//
// The scan is bound by instruction issue and the shared-memory gathers of
// the level table (one per dimension, the table replicated once per lane so
// a warp's gathers never conflict) about as tightly as by HBM. So:
//   * the work unit is one step of one tile: SBLK blocks (64 dims, or 128 for
//     odd rates, the shortest run of whole blocks ending on a 16-byte chunk
//     boundary) of 32 vectors, lane l decoding vector l. A CTA's tiles are cut
//     into units dealt round-robin to all its warps, so every warp streams
//     about the same number of units whatever the list lengths;
//   * each warp keeps a ring of its next units' codes in shared memory, filled
//     by bulk copies (chunk c of lane l of a tile at [tile][c][l], so a step of
//     a tile is one contiguous run) that complete on the slot's mbarrier;
//   * with V = 2 a unit covers the same step of two tiles, so each query value
//     read from shared memory serves two vectors per lane;
//   * each unit writes its 32 partial sums to shared memory; once a batch of
//     tiles is done, each tile's partials are summed in step order (so a
//     vector's distance does not depend on the schedule) and offered to the
//     warp's top-k, with the tiles' g1, h3 and ids already in shared memory
//     (bulk-copied when the batch starts);
//   * the level table sits in a static shared array, so its base folds into
//     the gathers' address; each digit's address is its field, shifted to the
//     entry stride, OR'ed with the lane's copy and the block's branch offset;
//   * the kernel is launched as a programmatic dependent of the routing
//     kernel: its barriers, query and table copies are set up while routing
//     finishes, and it reads the probes only after grid_dependency_wait().
//
// Reductions (the 16 warp lists of a CTA, then the CTAs' lists in the last
// CTA to finish): a list of the k best is reduced with a threshold filter
// and rank counting instead of a sort: T bounds the answer
// (the best of the lists' k-th entries, or the k-th best of their heads), so
// only entries <= T survive, and each survivor's rank among the survivors is
// its output slot. Ids are unique, so the ranks are distinct; when more than
// kSelCap entries survive (very small lists, large k) a block bitonic sort or
// a per-warp offer pass takes over.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "device_common.cuh"
#include "internal.h"
#include "decode_accum.cuh"
#include "scan_common.cuh"
#include "scan_plain.h"
#include "tma.cuh"

namespace e8qc {

namespace {

using namespace scan1;

// Level table copies of the rates whose [2][2^b] x copies fit 32 KB (b <=
// 12): a static array, so the gathers' base address is a constant.
constexpr int kStaticTab = 8192;
__shared__ __align__(128) float g_tab[kStaticTab];

template <int BITS>
__host__ __device__ constexpr bool static_tab() {
    return 2 * (1 << BITS) * table_rep(BITS) <= kStaticTab;
}

// Unit geometry: SBLK blocks in SCH chunks; odd rates end with an 8-block
// tail unit of TCH chunks when the block count leaves half a step.
template <int BITS, int V>
struct UnitGeo {
    static constexpr int SBLK = (BITS & 1) ? 16 : 8;
    static constexpr int SCH = SBLK * BITS / 16;
    static constexpr int TCH = (64 * BITS + 127) / 128;
};

// One block: 8 digits -> 8 gathers of this lane's table copy -> 8 FMAs.
// `lane4` = this lane's copy offset; the block's branch adds 2^b entries.
// Digit 7's stored LSB is the branch; its real LSB is the parity of digits
// 0..6 (bit SH of the XOR of the shifted fields: the lane and branch bits sit
// below and above it).
template <int BITS, int OFF>
__device__ __forceinline__ void block_fma_s(const uint32_t* w, const float* tab, uint32_t lane4, const float4 qa,
                                            const float4 qb, float& acc) {
    constexpr int SH = entry_shift(BITS);
    constexpr uint32_t L = 1u << SH;
    const uint32_t f7 = field_xs<OFF + 7 * BITS, BITS, SH>(w);
    const uint32_t lb = lane4 | ((f7 & L) << BITS);
    const uint32_t a0 = field_xs<OFF + 0 * BITS, BITS, SH>(w) | lb;
    const uint32_t a1 = field_xs<OFF + 1 * BITS, BITS, SH>(w) | lb;
    const uint32_t a2 = field_xs<OFF + 2 * BITS, BITS, SH>(w) | lb;
    const uint32_t a3 = field_xs<OFF + 3 * BITS, BITS, SH>(w) | lb;
    const uint32_t a4 = field_xs<OFF + 4 * BITS, BITS, SH>(w) | lb;
    const uint32_t a5 = field_xs<OFF + 5 * BITS, BITS, SH>(w) | lb;
    const uint32_t a6 = field_xs<OFF + 6 * BITS, BITS, SH>(w) | lb;
    const uint32_t par = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6;
    const uint32_t a7 = ((f7 & ~L) | (par & L)) | lb;
    const char* tb = reinterpret_cast<const char*>(tab);
    acc = __fmaf_rn(qa.x, *reinterpret_cast<const float*>(tb + a0), acc);
    acc = __fmaf_rn(qa.y, *reinterpret_cast<const float*>(tb + a1), acc);
    acc = __fmaf_rn(qa.z, *reinterpret_cast<const float*>(tb + a2), acc);
    acc = __fmaf_rn(qa.w, *reinterpret_cast<const float*>(tb + a3), acc);
    acc = __fmaf_rn(qb.x, *reinterpret_cast<const float*>(tb + a4), acc);
    acc = __fmaf_rn(qb.y, *reinterpret_cast<const float*>(tb + a5), acc);
    acc = __fmaf_rn(qb.z, *reinterpret_cast<const float*>(tb + a6), acc);
    acc = __fmaf_rn(qb.w, *reinterpret_cast<const float*>(tb + a7), acc);
}

// NBLK blocks of V vectors from their NCH register chunks each (vector v's
// chunks at buf[v * stride + c]); query blocks from q4 (2 float4 per block).
template <int BITS, int NBLK, int NCH, int V, int B0 = 0>
__device__ __forceinline__ void unit_fma(const uint32_t (&w)[V][4 * NCH + 1], const float* tab, uint32_t lane4,
                                         const float4* __restrict__ q4, float (&acc)[V][2]) {
    if constexpr (B0 < NBLK) {
        const float4 qa = q4[2 * B0], qb = q4[2 * B0 + 1];
#pragma unroll
        for (int v = 0; v < V; ++v) block_fma_s<BITS, B0 * 8 * BITS>(w[v], tab, lane4, qa, qb, acc[v][B0 & 1]);
        unit_fma<BITS, NBLK, NCH, V, B0 + 1>(w, tab, lane4, q4, acc);
    }
}

// Ring slots per warp (one unit's bulk copies each): as many as 120 KB of
// rings over the CTA's warps allow, 1 to 8 (a unit is V x SCH chunks of
// 512 B).
__host__ __device__ constexpr int ring_depth(int bits, int v) {
    return (122880 / (kWarps * v * (((bits & 1) ? 16 : 8) * bits / 16) * 512)) < 1
               ? 1
               : ((122880 / (kWarps * v * (((bits & 1) ? 16 : 8) * bits / 16) * 512)) > 8
                      ? 8
                      : 122880 / (kWarps * v * (((bits & 1) ? 16 : 8) * bits / 16) * 512));
}

__host__ __device__ constexpr bool static_tab_b(int bits) { return 2 * (1 << bits) * table_rep(bits) <= kStaticTab; }

// Byte offsets of the kernel's dynamic shared memory (host and device agree
// through this one function): the warps' unit rings, their mbarriers, the
// batch barrier and the test-hook barrier; the batch's g1 / h3 / ids rows (bulk-copy destinations,
// 128-byte aligned); [level table copies when not static]; query; tile
// offsets; the batch's tiles; unit partial sums; per-warp lists; survivors.
struct PlainCarve {
    size_t bars, meta, tab, query, off, tiles, part, lists, sel, total;
};
__host__ __device__ inline PlainCarve plain_carve(int bits, int v, int pd, int nunits, int tb) {
    PlainCarve c{};
    const int sch = ((bits & 1) ? 16 : 8) * bits / 16;
    const int ring = ring_depth(bits, v);
    size_t o = static_cast<size_t>(kWarps) * ring * v * sch * 512;
    c.bars = o;
    o += static_cast<size_t>(kWarps * ring + 2) * 8;
    o = (o + 127) & ~static_cast<size_t>(127);
    c.meta = o;
    o += static_cast<size_t>(tb + 1) * 32 * 4 * 3;
    c.tab = o;
    o += static_tab_b(bits) ? 0 : static_cast<size_t>(2) * (1 << bits) * table_rep(bits) * 4;
    c.query = o;
    o += static_cast<size_t>(pd) * 4;
    c.off = o;
    o += static_cast<size_t>(kToffCap + 4) * 4;
    c.tiles = o;
    o += static_cast<size_t>(tb + 1) * 12;
    o = (o + 15) & ~static_cast<size_t>(15);
    c.part = o;
    o += static_cast<size_t>(tb + 1) * nunits * 32 * 4;
    c.lists = o;
    o += static_cast<size_t>(kWarps) * kMaxK * 8;
    c.sel = o;
    o += static_cast<size_t>(kSelCap) * 8;
    c.total = o;
    return c;
}

template <int BITS, int V>
__global__ void __launch_bounds__(kWarps * 32, 1) scan_plain_kernel(
    DevIndex ix, const float* __restrict__ rq, RouteWork rw, int nprobe, int k, ScanWork sw, int tb_tiles,
    uint32_t* __restrict__ out_ids, float* __restrict__ out_d) {
    using U = UnitGeo<BITS, V>;
    constexpr int Q = 1 << BITS;
    constexpr int REP = table_rep(BITS);
    constexpr int SBLK = U::SBLK, SCH = U::SCH, TCH = U::TCH;
    constexpr int SLOT = V * SCH * 512;  // bytes of one unit's codes
    constexpr int kRing = ring_depth(BITS, V);
    constexpr bool kStatic = static_tab<BITS>();
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int nt = kWarps * 32;
    const int pd = ix.pd;
    const int nsteps = ix.B / SBLK;
    const bool tail = (ix.B % SBLK) != 0;  // odd rates: 8 blocks past the last full step
    const int nunits = nsteps + (tail ? 1 : 0);
    const PlainCarve cv = plain_carve(BITS, V, pd, nunits, tb_tiles);
    unsigned char* ring = smem;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + cv.bars);  // kWarps*kRing ring slots, then the batch's
    uint64_t* bbar = bars + kWarps * kRing;
    uint64_t* sbar = bbar + 1;  // the test hook's barrier (nothing completes it)
    float* s_g1 = reinterpret_cast<float*>(smem + cv.meta);  // (tb_tiles + 1) * 32 each
    float* s_h3 = s_g1 + (tb_tiles + 1) * 32;
    uint32_t* s_ids = reinterpret_cast<uint32_t*>(s_h3 + (tb_tiles + 1) * 32);
    float* tab = kStatic ? g_tab : reinterpret_cast<float*>(smem + cv.tab);
    float* sq = reinterpret_cast<float*>(smem + cv.query);
    uint32_t* soff = reinterpret_cast<uint32_t*>(smem + cv.off);
    uint32_t* s_gt = reinterpret_cast<uint32_t*>(smem + cv.tiles);  // tb_tiles + 1 each
    float* s_d2 = reinterpret_cast<float*>(s_gt + tb_tiles + 1);
    uint32_t* s_nv = reinterpret_cast<uint32_t*>(s_d2 + tb_tiles + 1);
    float* part = reinterpret_cast<float*>(smem + cv.part);
    float* sm_d = reinterpret_cast<float*>(smem + cv.lists);  // kWarps * kMaxK
    uint32_t* sm_id = reinterpret_cast<uint32_t*>(sm_d + kWarps * kMaxK);
    float* sv_d = reinterpret_cast<float*>(smem + cv.sel);  // kSelCap
    uint32_t* sv_id = reinterpret_cast<uint32_t*>(sv_d + kSelCap);
    __shared__ bool s_last;

    // ---- setup that does not read the routing launch's results: with a
    // programmatic launch it overlaps the routing kernel's tail
    if (tid == 0) {
        for (int b = 0; b < kWarps * kRing + 2; ++b) mbar_init(bars + b, 1);
        fence_barrier_init();
        if (sw.stuck_ms != 0 && blockIdx.x == 0) {
            // test hook: a wait on a barrier nothing completes, bounded like
            // every wait here; giving up is recorded as a wait timeout, then
            // the phase is completed so the barrier can be invalidated
            if (!mbar_wait_bounded(sbar, 0u, sw.stuck_ms)) atomicOr(sw.err, kErrWaitTimeout);
            mbar_arrive(sbar);
        }
    }
    for (int i = tid; i < pd; i += nt) sq[i] = rq[i];
    // one load per table entry, then its per-lane copies
    for (int e = tid; e < 2 * Q; e += nt) {
        const float v = __ldg(ix.tab + e);
#pragma unroll 8
        for (int c = 0; c < REP; ++c) tab[e * REP + c] = v;
    }
    grid_dependency_wait();
    const bool off_in_smem = nprobe <= kToffCap;
    if (off_in_smem)
        for (int i = tid; i <= nprobe; i += nt) soff[i] = __ldcg(rw.tile_off + i);
    __syncthreads();
    const uint32_t* off = off_in_smem ? soff : rw.tile_off;
    const float4* sq4 = reinterpret_cast<const float4*>(sq);
    const uint32_t lane4 = static_cast<uint32_t>(lane % REP) * 4u;  // this lane's table copy
    const uint32_t T = __ldcg(rw.total_tiles);
    const uint32_t Gd = gridDim.x;
    const uint32_t per_cta = T > blockIdx.x ? (T - blockIdx.x + Gd - 1) / Gd : 0;
    unsigned char* my_ring = ring + warp * kRing * SLOT;
    uint64_t* my_bars = bars + warp * kRing;
    uint32_t seq = 0;  // this warp's units so far (ring slot = seq % kRing, parity = (seq / kRing) & 1)
    uint32_t batch_no = 0;

    WarpTopK top;
    top.init(k);
    for (uint32_t jb = 0; jb < per_cta; jb += static_cast<uint32_t>(tb_tiles), ++batch_no) {
        const int nb = static_cast<int>(min(static_cast<uint32_t>(tb_tiles), per_cta - jb));
        // the batch's tiles: global tile, probe d2, vectors present; a
        // missing partner of the last pair (V = 2) reads tile 0 of the batch
        // into the spare row
        for (int j = tid; j <= nb; j += nt) {
            const int jj = j < nb ? j : 0;
            const uint32_t t = blockIdx.x + (jb + jj) * Gd;
            const int p = find_probe(off, nprobe, t);
            const uint2 info = __ldcg(rw.probe_info + p);
            const uint32_t local = t - off[p];
            s_gt[j] = info.x + local;
            s_d2[j] = __ldcg(rw.probe_d2 + p);
            s_nv[j] = j < nb ? min(32u, info.y - local * 32u) : 0u;
        }
        __syncthreads();
        // the epilogue's g1, h3 and ids of the batch's tiles (128 contiguous
        // bytes each per tile), copied in the background on the batch barrier
        if (warp == 0) {
            fence_proxy_async_smem();
            if (lane == 0) mbar_arrive_expect_tx(bbar, static_cast<uint32_t>(nb) * 384u);
            __syncwarp();
            for (int j = lane; j < nb; j += 32) {
                const size_t o = static_cast<size_t>(s_gt[j]) * 32u;
                bulk_g2s(s_g1 + j * 32, ix.g1 + o, 128u, bbar);
                bulk_g2s(s_h3 + j * 32, ix.h3 + o, 128u, bbar);
                bulk_g2s(s_ids + j * 32, ix.ids + o, 128u, bbar);
            }
        }
        const int ngroups = (nb + V - 1) / V;
        const int nu = ngroups * nunits;  // units of this batch: (tile group g, step st)
        // lane 0 puts unit u's codes (V tiles x the step's chunks, contiguous
        // per tile) in ring slot r with one bulk copy per tile
        auto issue = [&](int u, int g, int st, uint32_t sq_no) {
            if (lane == 0 && u < nu) {
                const int r = static_cast<int>(sq_no % kRing);
                const uint32_t bytes = static_cast<uint32_t>((st < nsteps ? SCH : TCH) * 512);
                mbar_arrive_expect_tx(my_bars + r, bytes * V);
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    const int j = g * V + v < nb ? g * V + v : nb;
                    const uint4* src = ix.codes + (static_cast<size_t>(s_gt[j]) * ix.nch +
                                                   static_cast<size_t>(st) * SCH) * 32;
                    bulk_g2s(my_ring + r * SLOT + v * SCH * 512, src, bytes, my_bars + r);
                }
            }
        };
        // this warp's units u = warp + kWarps * i, walked with (g, st)
        int u_is = warp, g_is = warp / nunits, st_is = warp - g_is * nunits;  // issue cursor
        auto advance = [&](int& u_, int& g_, int& st_) {
            u_ += kWarps;
            st_ += kWarps;
            while (st_ >= nunits) {
                st_ -= nunits;
                ++g_;
            }
        };
        uint32_t seq_is = seq;
#pragma unroll
        for (int r = 0; r < kRing - 1; ++r) {
            issue(u_is, g_is, st_is, seq_is);
            if (u_is < nu) ++seq_is;
            advance(u_is, g_is, st_is);
        }
        int g = warp / nunits, st = warp - (warp / nunits) * nunits;
        for (int u = warp; u < nu; u += kWarps) {
            issue(u_is, g_is, st_is, seq_is);
            if (u_is < nu) ++seq_is;
            advance(u_is, g_is, st_is);
            const int r = static_cast<int>(seq % kRing);
            if (!mbar_wait_bounded(my_bars + r, (seq / kRing) & 1u, 2000u)) {
                // a bulk copy that did not land: report it, and give the copy
                // one more bounded wait so it is not left writing into shared
                // memory after the CTA moves on
                if (lane == 0) atomicOr(sw.err, kErrWaitTimeout);
                (void)mbar_wait_bounded(my_bars + r, (seq / kRing) & 1u, 2000u);
            }
            ++seq;
            const uint4* slot = reinterpret_cast<const uint4*>(my_ring + r * SLOT) + lane;
            uint32_t w[V][4 * SCH + 1];
#pragma unroll
            for (int v = 0; v < V; ++v) {
#pragma unroll
                for (int c = 0; c < SCH; ++c) {
                    const uint4 x = slot[(v * SCH + c) * 32];
                    w[v][4 * c] = x.x;
                    w[v][4 * c + 1] = x.y;
                    w[v][4 * c + 2] = x.z;
                    w[v][4 * c + 3] = x.w;
                }
                w[v][4 * SCH] = 0u;
            }
            float acc[V][2];
#pragma unroll
            for (int v = 0; v < V; ++v) acc[v][0] = acc[v][1] = 0.0f;
            if (st < nsteps) {
                unit_fma<BITS, SBLK, SCH, V>(w, tab, lane4, sq4 + 2 * st * SBLK, acc);
            } else if constexpr ((BITS & 1) != 0) {
                unit_fma<BITS, 8, SCH, V>(w, tab, lane4, sq4 + 2 * st * SBLK, acc);
            }
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int j = g * V + v < nb ? g * V + v : nb;
                part[(j * nunits + st) * 32 + lane] = __fadd_rn(acc[v][0], acc[v][1]);
            }
            // every lane has consumed the slot before lane 0 refills it
            __syncwarp();
            advance(u, g, st);
            u -= kWarps;  // the for-loop adds it back
        }
        __syncthreads();
        if (!mbar_wait_bounded(bbar, batch_no & 1u, 2000u)) {
            if (tid == 0) atomicOr(sw.err, kErrWaitTimeout);
            (void)mbar_wait_bounded(bbar, batch_no & 1u, 2000u);
        }
        // each tile's partials in step order, then the estimator
        for (int j = warp; j < nb; j += kWarps) {
            float S = 0.0f;
            for (int s2 = 0; s2 < nunits; ++s2) S = __fadd_rn(S, part[(j * nunits + s2) * 32 + lane]);
            const float g1 = s_g1[j * 32 + lane], h3 = s_h3[j * 32 + lane];
            const float dist = __fmaf_rn(-__fmul_rn(2.0f, g1), S, __fadd_rn(s_d2[j], h3));
            const uint32_t id = s_ids[j * 32 + lane];
            top.offer(dist, static_cast<uint32_t>(lane) < s_nv[j], [&] { return id; });
        }
        __syncthreads();
    }

    // the rings are idle: their barriers give the space back to plain data
    if (tid == 0)
        for (int b = 0; b < kWarps * kRing + 2; ++b) mbar_inval(bars + b);
    // CTA reduction of the warps' lists
    top.store(sm_d + warp * k, sm_id + warp * k, k);
    __syncthreads();
    float* cta_d = sw.part_d + static_cast<size_t>(blockIdx.x) * kMaxK;
    uint32_t* cta_id = sw.part_id + static_cast<size_t>(blockIdx.x) * kMaxK;
    if (!block_select(sm_d, sm_id, kWarps, k, sv_d, sv_id, cta_d, cta_id)) {
        __syncthreads();
        block_sort_select(sm_d, sm_id, kWarps, k, cta_d, cta_id);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(sw.counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();

    // final reduction over the per-CTA lists: staged in shared memory (the
    // rings, table copies and partials are free now) when they fit
    const int Gi = static_cast<int>(gridDim.x);
    const int room = static_cast<int>(cv.lists / 8);  // entries that fit below the warp lists
    float* st_d = reinterpret_cast<float*>(smem);
    uint32_t* st_i = reinterpret_cast<uint32_t*>(smem) + (Gi * k);
    bool done = false;
    if (Gi * k <= room) {
        for (int e = tid; e < Gi * k; e += nt) {
            const int c = e / k, jj = e - c * k;
            st_d[e] = __ldcg(sw.part_d + static_cast<size_t>(c) * kMaxK + jj);
            st_i[e] = __ldcg(sw.part_id + static_cast<size_t>(c) * kMaxK + jj);
        }
        __syncthreads();
        done = block_select(st_d, st_i, Gi, k, sv_d, sv_id, out_d, out_ids);
        __syncthreads();
        if (!done && 2 * next_pow2(Gi * k) <= room) {
            // many entries tie or beat the threshold: sort them all
            float* bd = reinterpret_cast<float*>(smem);
            uint32_t* bi = reinterpret_cast<uint32_t*>(smem) + next_pow2(Gi * k);
            for (int e = tid; e < Gi * k; e += nt) {
                const int c = e / k, jj = e - c * k;
                bd[e] = __ldcg(sw.part_d + static_cast<size_t>(c) * kMaxK + jj);
                bi[e] = __ldcg(sw.part_id + static_cast<size_t>(c) * kMaxK + jj);
            }
            __syncthreads();
            block_sort_select(bd, bi, Gi, k, out_d, out_ids);
            done = true;
        }
    }
    if (!done) {
        // many survivors or lists too large to stage: each warp folds a share
        // of the per-CTA lists into its top-k, then the warps' lists reduce
        top.init(k);
        for (int e0 = warp * 32; e0 < Gi * k; e0 += kWarps * 32) {
            const int e = e0 + lane;
            const bool okj = e < Gi * k;
            float dd = inf_f();
            uint32_t ii = 0xFFFFFFFFu;
            if (okj) {
                const int c = e / k, jj = e - c * k;
                dd = __ldcg(sw.part_d + static_cast<size_t>(c) * kMaxK + jj);
                ii = __ldcg(sw.part_id + static_cast<size_t>(c) * kMaxK + jj);
            }
            top.offer_pair(dd, ii, okj && ii != 0xFFFFFFFFu);
        }
        top.store(sm_d + warp * k, sm_id + warp * k, k);
        __syncthreads();
        if (!block_select(sm_d, sm_id, kWarps, k, sv_d, sv_id, out_d, out_ids)) {
            __syncthreads();
            block_sort_select(sm_d, sm_id, kWarps, k, out_d, out_ids);
        }
    }
    if (tid == 0) *sw.counter = 0;
}

template <int BITS, int V>
int launch_bits(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k, const ScanWork& sw,
                const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s) {
    const size_t smem = geo.smem;
    // dynamic shared-memory opt-in, raised per device as needed
    static size_t configured[64] = {};
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    if (configured[dev & 63] < smem) {
        E8QC_CUDA(cudaFuncSetAttribute(scan_plain_kernel<BITS, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        configured[dev & 63] = smem;
    }
    // a programmatic dependent of the routing launch before it: the setup
    // that does not read the routing results runs while routing finishes
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(sw.grid));
    cfg.blockDim = dim3(kWarps * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    E8QC_CUDA(cudaLaunchKernelEx(&cfg, scan_plain_kernel<BITS, V>, ix, rq, rw, nprobe, k, sw, geo.tb_tiles, out_ids,
                                 out_d));
    return 1;
}

template <int BITS>
int launch_v(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k, const ScanWork& sw,
             const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s) {
    if (geo.v == 2) return launch_bits<BITS, 2>(ix, rq, rw, nprobe, k, sw, geo, out_ids, out_d, s);
    return launch_bits<BITS, 1>(ix, rq, rw, nprobe, k, sw, geo, out_ids, out_d, s);
}

}  // namespace

size_t scan_smem_bytes(const DevIndex& ix, int tb_tiles, int v) {
    const int sblk = (ix.bits & 1) ? 16 : 8;
    const int nunits = ix.B / sblk + ((ix.B % sblk) ? 1 : 0);
    return plain_carve(ix.bits, v, ix.pd, nunits, tb_tiles).total;
}

ScanGeo plain_scan_geo(const DevIndex& ix, size_t max_tiles_per_cta) {
    ScanGeo g{};
    g.warps = kWarps;
    // two vectors per lane per unit (each query value read from shared
    // memory serves two tiles) where the wider ring still holds two units
    // per warp; tiles per batch: the partial sums of up to 64 tiles (no more
    // than a CTA gets), within the shared-memory budget (the static table
    // takes up to 32 KB beside it)
    const size_t budget = 190 * 1024;
    g.v = ring_depth(ix.bits, 2) >= 2 ? 2 : 1;
    const int want = static_cast<int>(
        std::min<size_t>(64, std::max<size_t>(2, max_tiles_per_cta + (max_tiles_per_cta & 1))));
    g.tb_tiles = want;
    while (g.tb_tiles > 2 && scan_smem_bytes(ix, g.tb_tiles, g.v) > budget) g.tb_tiles -= 2;
    if (g.v == 2 && scan_smem_bytes(ix, g.tb_tiles, g.v) > budget) {
        g.v = 1;
        g.tb_tiles = want;
        while (g.tb_tiles > 2 && scan_smem_bytes(ix, g.tb_tiles, g.v) > budget) g.tb_tiles -= 2;
    }
    g.smem = scan_smem_bytes(ix, g.tb_tiles, g.v);
    return g;
}

int launch_scan_plain(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k,
                      const ScanWork& sw, const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s) {
    if (geo.smem + kStaticTab * 4 + 1024 > 227 * 1024)
        fail(E8QC_EINVAL, "padded dimension too large for the plain scan's shared memory");
    switch (ix.bits) {
#define E8QC_CASE(b) \
    case b: return launch_v<b>(ix, rq, rw, nprobe, k, sw, geo, out_ids, out_d, s);
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    return 0;
}

}  // namespace e8qc
