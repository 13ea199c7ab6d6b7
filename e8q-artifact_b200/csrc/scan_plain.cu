// Plain one-query streaming scan (the drop-in search path).
//
// Every vector of every probed list gets the exact estimator
//   dist = (d2 + h3) - 2*g1*S,   S = sum_i q[i] * level[branch][digit_i] / sqrt(D)
// (src/simd/e8q_search_generic.cpp:58-66 with d2 folded as at :189) and enters
// a warp top-k; each CTA reduces its warps' lists to one, and the last CTA to
// finish reduces the per-CTA lists to the answer.
//
// The scan is bound by HBM and, nearly as tightly, by instruction issue and
// the shared-memory gathers of the level table (one per dimension, the table
// replicated once per lane so a warp's gathers never conflict). So:
//   * the work unit is one step of one tile: SBLK blocks (64 dims, or 128 for
//     odd rates, the shortest run of whole blocks ending on a 16-byte chunk
//     boundary) of 32 vectors, lane l decoding vector l. A CTA's tiles are cut
//     into units dealt round-robin to all its warps, so every warp streams
//     about the same number of units whatever the list lengths;
//   * a warp streams its units' codes straight from HBM into registers through
//     a ring R units deep (chunk c of lane l of a tile at [tile][c][l]: one
//     16-byte load per lane reads 512 contiguous bytes); nothing is staged;
//   * with V = 2 a unit covers the same step of two tiles, so each query value
//     read from shared memory serves two vectors per lane;
//   * each unit writes its 32 partial sums to shared memory; once a batch of
//     tiles is done, each tile's partials are summed in step order (so a
//     vector's distance does not depend on the schedule) and offered to the
//     warp's top-k;
//   * the level table sits in a static shared array, so its base folds into
//     the gathers' address; each digit's address is its field, shifted to the
//     entry stride, OR'ed with the lane's copy and the block's branch offset.
//
// Reductions: a list of the k best is reduced with a threshold filter and
// rank counting instead of a sort: T = the best of the lists' k-th entries
// bounds the answer (the list holding T has k entries <= T), so only entries
// <= T survive, and each survivor's rank among the survivors is its output
// slot. Ids are unique, so the ranks are distinct; when more than kSelCap
// entries survive (very small lists, large k) a block bitonic sort or a
// per-warp offer pass takes over.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include "device_common.cuh"
#include "internal.h"
#include "decode_accum.cuh"
#include "scan_common.cuh"
#include "scan_plain.h"

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
// tail unit of TCH chunks when the block count leaves half a step; R units in
// flight per warp (V vectors per lane each).
template <int BITS, int V>
struct UnitGeo {
    static constexpr int SBLK = (BITS & 1) ? 16 : 8;
    static constexpr int SCH = SBLK * BITS / 16;
    static constexpr int TCH = (64 * BITS + 127) / 128;
    static constexpr int R = (V * SCH <= 3) ? 4 : (V * SCH <= 6 ? 3 : (V * SCH <= 8 ? 2 : 1));
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

template <int BITS, int V>
__global__ void __launch_bounds__(kWarps * 32, 1) scan_plain_kernel(
    DevIndex ix, const float* __restrict__ rq, RouteWork rw, int nprobe, int k, ScanWork sw, int tb_tiles,
    uint32_t* __restrict__ out_ids, float* __restrict__ out_d) {
    using U = UnitGeo<BITS, V>;
    constexpr int Q = 1 << BITS;
    constexpr int REP = table_rep(BITS);
    constexpr int SBLK = U::SBLK, SCH = U::SCH, TCH = U::TCH, R = U::R;
    constexpr bool kStatic = static_tab<BITS>();
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int nt = kWarps * 32;
    const int pd = ix.pd;
    const int nsteps = ix.B / SBLK;
    const bool tail = (ix.B % SBLK) != 0;  // odd rates: 8 blocks past the last full step
    const int nunits = nsteps + (tail ? 1 : 0);
    // shared-memory carve (scan_smem_bytes): [level table copies when not
    // static], query, tile offsets, the batch's tiles, unit partial sums,
    // per-warp lists, survivors
    float* tab = kStatic ? g_tab : reinterpret_cast<float*>(smem);
    float* sq = reinterpret_cast<float*>(smem) + (kStatic ? 0 : 2 * Q * REP);  // pd
    uint32_t* soff = reinterpret_cast<uint32_t*>(sq + pd);                       // kToffCap + 4
    uint32_t* s_gt = soff + kToffCap + 4;                                         // tb_tiles + 1
    float* s_d2 = reinterpret_cast<float*>(s_gt + tb_tiles + 1);                 // tb_tiles + 1
    uint32_t* s_nv = reinterpret_cast<uint32_t*>(s_d2 + tb_tiles + 1);           // tb_tiles + 1
    float* part = reinterpret_cast<float*>(s_nv + tb_tiles + 1);                 // (tb_tiles + 1) * nunits * 32
    float* sm_d = part + (tb_tiles + 1) * nunits * 32;                           // kWarps * kMaxK
    uint32_t* sm_id = reinterpret_cast<uint32_t*>(sm_d + kWarps * kMaxK);
    float* sv_d = reinterpret_cast<float*>(sm_id + kWarps * kMaxK);             // kSelCap
    uint32_t* sv_id = reinterpret_cast<uint32_t*>(sv_d + kSelCap);
    __shared__ bool s_last;

    for (int i = tid; i < pd; i += nt) sq[i] = rq[i];
    for (int e = tid; e < 2 * Q * REP; e += nt) tab[e] = ix.tab[e / REP];
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

    WarpTopK top;
    top.init(k);
    for (uint32_t jb = 0; jb < per_cta; jb += static_cast<uint32_t>(tb_tiles)) {
        const int nb = static_cast<int>(min(static_cast<uint32_t>(tb_tiles), per_cta - jb));
        // the batch's tiles: global tile, probe d2, vectors present; a
        // missing partner of the last pair (V = 2) reads tile 0 of the batch
        // into the spare row
        for (int j = tid; j <= nb; j += nt) {
            const int jj = j < nb ? j : 0;
            const uint32_t t = blockIdx.x + (jb + jj) * Gd;
            const int p = find_probe(off, nprobe, t);
            const uint32_t list = __ldcg(rw.probes + p);
            const uint32_t local = t - off[p];
            s_gt[j] = __ldg(ix.tile_begin + list) + local;
            s_d2[j] = __ldcg(rw.probe_d2 + p);
            s_nv[j] = j < nb ? min(32u, __ldg(ix.list_len + list) - local * 32u) : 0u;
        }
        __syncthreads();
        const int ngroups = (nb + V - 1) / V;
        const int nu = ngroups * nunits;  // units of this batch
        // unit u: tiles g*V .. g*V+V-1 (g = u / nunits), step s = u % nunits
        auto unit_src = [&](int u, int v) -> const uint4* {
            const int g = u / nunits, st = u - g * nunits;
            const int j = g * V + v < nb ? g * V + v : nb;
            return ix.codes + (static_cast<size_t>(s_gt[j]) * ix.nch + static_cast<size_t>(st) * SCH) * 32 + lane;
        };
        uint4 buf[R][V][SCH];
        auto load_unit = [&](int slot_r, int u) {
            const int st = u % nunits;
            const int cnt = st < nsteps ? SCH : TCH;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const uint4* src = unit_src(u, v);
#pragma unroll
                for (int c = 0; c < SCH; ++c)
                    if (c < cnt) buf[slot_r][v][c] = ld_stream(src + c * 32);
            }
        };
        int u = warp;
#pragma unroll
        for (int r = 0; r < R - 1; ++r)
            if (u + r * kWarps < nu) load_unit(r, u + r * kWarps);
        for (; u < nu; u += R * kWarps) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int uu = u + r * kWarps;
                if (uu < nu) {
                    const int un = uu + (R - 1) * kWarps;
                    if (un < nu) load_unit((r + R - 1) % R, un);
                    const int g = uu / nunits, st = uu - g * nunits;
                    uint32_t w[V][4 * SCH + 1];
#pragma unroll
                    for (int v = 0; v < V; ++v) {
#pragma unroll
                        for (int c = 0; c < SCH; ++c) {
                            w[v][4 * c] = buf[r][v][c].x;
                            w[v][4 * c + 1] = buf[r][v][c].y;
                            w[v][4 * c + 2] = buf[r][v][c].z;
                            w[v][4 * c + 3] = buf[r][v][c].w;
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
                }
            }
        }
        __syncthreads();
        // each tile's partials in step order, then the estimator
        for (int j = warp; j < nb; j += kWarps) {
            float S = 0.0f;
            for (int st = 0; st < nunits; ++st) S = __fadd_rn(S, part[(j * nunits + st) * 32 + lane]);
            const size_t slot = static_cast<size_t>(s_gt[j]) * 32u + lane;
            const float g1 = __ldg(ix.g1 + slot), h3 = __ldg(ix.h3 + slot);
            const float dist = __fmaf_rn(-__fmul_rn(2.0f, g1), S, __fadd_rn(s_d2[j], h3));
            top.offer(dist, static_cast<uint32_t>(lane) < s_nv[j], [&] { return __ldg(ix.ids + slot); });
        }
        __syncthreads();
    }

    // CTA reduction of the warps' lists (part-1 warps hold only padding)
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
    // table and query space is free now) when they fit
    const int Gi = static_cast<int>(gridDim.x);
    float* st_d = reinterpret_cast<float*>(smem);
    uint32_t* st_i = reinterpret_cast<uint32_t*>(smem) + (Gi * k);  // the query, offsets and partials are free now
    bool done = false;
    if (Gi * k <= static_cast<int>((reinterpret_cast<unsigned char*>(sm_d) - smem) / 8)) {
        for (int e = tid; e < Gi * k; e += nt) {
            const int c = e / k, jj = e - c * k;
            st_d[e] = __ldcg(sw.part_d + static_cast<size_t>(c) * kMaxK + jj);
            st_i[e] = __ldcg(sw.part_id + static_cast<size_t>(c) * kMaxK + jj);
        }
        __syncthreads();
        done = block_select(st_d, st_i, Gi, k, sv_d, sv_id, out_d, out_ids);
        __syncthreads();
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
    scan_plain_kernel<BITS, V><<<sw.grid, kWarps * 32, smem, s>>>(ix, rq, rw, nprobe, k, sw, geo.tb_tiles, out_ids,
                                                                  out_d);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

template <int BITS>
int launch_v(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k, const ScanWork& sw,
             const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s) {
    if (geo.v == 2) return launch_bits<BITS, 2>(ix, rq, rw, nprobe, k, sw, geo, out_ids, out_d, s);
    return launch_bits<BITS, 1>(ix, rq, rw, nprobe, k, sw, geo, out_ids, out_d, s);
}

}  // namespace

size_t scan_smem_bytes(const DevIndex& ix, int tb_tiles) {
    const int q = 1 << ix.bits;
    const int sblk = (ix.bits & 1) ? 16 : 8;
    const int nunits = ix.B / sblk + ((ix.B % sblk) ? 1 : 0);
    const bool stat = 2 * q * table_rep(ix.bits) <= kStaticTab;
    size_t b = stat ? 0 : static_cast<size_t>(2) * q * table_rep(ix.bits) * 4;
    b += static_cast<size_t>(ix.pd) * 4;
    b += static_cast<size_t>(kToffCap + 4) * 4;
    b += static_cast<size_t>(tb_tiles + 1) * 12;
    b += static_cast<size_t>(tb_tiles + 1) * nunits * 32 * 4;
    b += static_cast<size_t>(kWarps) * kMaxK * 8;
    b += static_cast<size_t>(kSelCap) * 8;
    return b;
}

ScanGeo plain_scan_geo(const DevIndex& ix) {
    ScanGeo g{};
    g.warps = kWarps;
    g.v = 1;
    if (const char* e = getenv("E8QC_PLAIN_V")) {
        if (e[0] == '2') g.v = 2;
    }
    // tiles per batch: the partial sums of up to 64 tiles, within the
    // shared-memory budget (the static table takes up to 32 KB of it)
    const size_t budget = 190 * 1024;
    g.tb_tiles = 64;
    while (g.tb_tiles > 2 && scan_smem_bytes(ix, g.tb_tiles) > budget) g.tb_tiles -= 2;
    g.smem = scan_smem_bytes(ix, g.tb_tiles);
    return g;
}

int launch_scan_plain(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k,
                      const ScanWork& sw, const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s) {
    if (geo.smem + kStaticTab * 4 > 227 * 1024)
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
