// Plain one-query streaming scan (the drop-in search path).
//
// Every vector of every probed list gets the exact estimator
//   dist = (d2 + h3) - 2*g1*S,   S = sum_i q[i] * level[branch][digit_i] / sqrt(D)
// (src/simd/e8q_search_generic.cpp:58-66 with d2 folded as at :189) and enters
// a warp top-k; CTAs merge into per-CTA lists and the last CTA to finish
// merges those into the answer.
//
// Data movement: lane l decodes vector l of a 32-vector tile; chunk c of lane
// l sits at [c][l] (16 bytes), so a warp's read of one chunk row is 512
// contiguous bytes. Each warp runs a kStages-deep cp.async pipeline over its
// jobs (one chunk-group of a tile each): every lane copies exactly the 16-byte
// entries it will decode into the warp's ring slot, so completion is a plain
// per-thread cp.async.wait_group (no spinning, no cross-lane hand-off). Level
// values come from a shared-memory table replicated once per lane
// (bank-conflict-free gathers). Tiles are dealt round-robin over CTAs.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "internal.h"
#include "decode_accum.cuh"
#include "scan_plain.h"

namespace e8qc {

namespace {

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

constexpr int kMaxWarps = 16;
constexpr int kStages = 4;      // cp.async stages in flight per warp
constexpr int kParts = 4;       // warps sharing one tile
constexpr int kToffCap = 1024;  // tile offsets cached in shared memory

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte global -> shared async copy (L2 only), and the group fences.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
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

// CTA-wide merge of the per-warp top-k lists: all lists into shared memory,
// one block bitonic sort, warp 0 reloads the first k (sm_d/sm_id hold
// nw*kMaxK >= next_pow2(nw*k) entries).
__device__ void cta_merge(WarpTopK& top, float* sm_d, uint32_t* sm_id, int k) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    top.store(sm_d + warp * k, sm_id + warp * k, k);
    const int n = nw * k, pn = next_pow2(n);
    for (int i = n + threadIdx.x; i < pn; i += blockDim.x) {
        sm_d[i] = inf_f();
        sm_id[i] = 0xFFFFFFFFu;
    }
    __syncthreads();
    block_bitonic_sort(sm_d, sm_id, pn);
    if (warp == 0) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int j = s * 32 + lane;
            top.d[s] = j < k ? sm_d[j] : inf_f();
            top.id[s] = j < k ? sm_id[j] : 0xFFFFFFFFu;
        }
        top.refresh_threshold();
    }
    __syncthreads();
}

// Where one tile of the warp's share lives and what its epilogue needs.
struct TileInfo {
    const uint4* src;  // first chunk row of the tile
    float d2;          // query-to-list distance
    uint32_t slot0;    // first padded slot of the tile
    uint32_t nvalid;   // vectors of the tile that exist (<= 32)
};

template <int BITS>
__global__ void __launch_bounds__(kMaxWarps * 32, 1) scan_plain_kernel(
    DevIndex ix, const float* __restrict__ rq, RouteWork rw, int nprobe, int k, ScanWork sw, ScanGeo geo,
    uint32_t* __restrict__ out_ids, float* __restrict__ out_d) {
    constexpr int GBL = group_blocks(BITS), GCH = group_chunks(BITS);
    constexpr int TCH = (64 * BITS + 127) / 128;
    constexpr int Q = 1 << BITS;
    constexpr int REP = table_rep(BITS);
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nw = blockDim.x >> 5, nt = blockDim.x;
    const int pd = ix.pd;
    // shared-memory carve (see scan_smem_bytes)
    unsigned char* ring = smem;                                       // nw * kStages * seg_bytes
    float* tabrep = reinterpret_cast<float*>(ring + nw * kStages * geo.seg_bytes);  // 2*Q*REP
    float* sq = tabrep + 2 * Q * REP;                                 // pd
    uint32_t* soff = reinterpret_cast<uint32_t*>(sq + pd);           // kToffCap + 1
    float* sm_d = reinterpret_cast<float*>(soff + kToffCap + 1);      // nw * kMaxK
    uint32_t* sm_id = reinterpret_cast<uint32_t*>(sm_d + nw * kMaxK);
    float* spart = reinterpret_cast<float*>(sm_id + nw * kMaxK);     // 2 * nw * 32
    __shared__ bool s_last;

    for (int i = tid; i < pd; i += nt) sq[i] = rq[i];
    for (int e = tid; e < 2 * Q * REP; e += nt) tabrep[e] = ix.tab[e / REP];
    const bool off_in_smem = nprobe <= kToffCap;
    if (off_in_smem)
        for (int i = tid; i <= nprobe; i += nt) soff[i] = __ldcg(rw.tile_off + i);
    __syncthreads();
    const uint32_t* off = off_in_smem ? soff : rw.tile_off;
    const float4* sq4 = reinterpret_cast<const float4*>(sq);
    // byte address of this lane's table copy (entry e at e*REP*4 + copy*4)
    const uint32_t tb_addr = smem_addr(tabrep) + static_cast<uint32_t>(lane % REP) * 4u;
    const uint32_t T = __ldcg(rw.total_tiles);
    // tiles dealt round-robin over CTAs, then over the CTA's tile groups; a
    // group of `parts` warps shares each tile, warp `pi` decoding a contiguous
    // range of its chunk-groups
    const uint32_t G = gridDim.x;
    const uint32_t per_cta = T > blockIdx.x ? (T - blockIdx.x + G - 1) / G : 0;
    const int parts = nw < kParts ? nw : kParts;
    const int ngrp = nw / parts;
    const int gi = warp / parts, pi = warp % parts;
    const uint32_t ntile_g = per_cta > static_cast<uint32_t>(gi)
                                 ? (per_cta - gi + ngrp - 1) / static_cast<uint32_t>(ngrp) : 0;
    const int jpt = geo.ng + geo.tail;  // chunk-group jobs per tile
    const int j_lo = (pi * jpt) / parts, j_hi = ((pi + 1) * jpt) / parts;
    const int jmine = j_hi - j_lo;
    const uint32_t J = ntile_g * static_cast<uint32_t>(jmine);
    // per-warp ring of kStages chunk-group slots; lane l copies and later
    // reads only its own 16-byte entries, so the pipeline is lane-private
    const uint32_t ring_lane = smem_addr(ring) + static_cast<uint32_t>(warp * kStages * geo.seg_bytes) +
                               static_cast<uint32_t>(lane) * 16u;
    auto tile_of = [&](uint32_t i) { return (static_cast<uint32_t>(gi) + i * ngrp) * G + blockIdx.x; };
    // every lane resolves the same tile (broadcast loads, no divergence)
    auto resolve = [&](uint32_t i) {
        TileInfo ti{nullptr, 0.0f, 0u, 0u};
        if (i >= ntile_g) return ti;
        const uint32_t t = tile_of(i);
        const int p = find_probe(off, nprobe, t);
        const uint32_t list = __ldcg(rw.probes + p);
        const uint32_t local = t - off[p];
        const uint32_t gt = __ldg(ix.tile_begin + list) + local;
        const uint32_t len = __ldg(ix.list_len + list);
        ti.src = ix.codes + static_cast<size_t>(gt) * ix.nch * 32;
        ti.d2 = __ldcg(rw.probe_d2 + p);
        ti.slot0 = gt * 32u;
        ti.nvalid = min(32u, len - local * 32u);
        return ti;
    };
    // the issue side walks the jobs ahead of the consume side with its own
    // tile cursor; both resolve a tile once (broadcast loads)
    uint32_t iss_i = 0xFFFFFFFFu;
    TileInfo iss{nullptr, 0.0f, 0u, 0u};
    auto issue = [&](uint32_t j) {
        if (j < J) {
            const uint32_t i = j / jmine;
            if (i != iss_i) {
                iss_i = i;
                iss = resolve(i);
            }
            const int g = j_lo + static_cast<int>(j % jmine);
            const int c0 = g * GCH;
            const int cnt = g < geo.ng ? GCH : TCH;
            const uint32_t dst = ring_lane + static_cast<uint32_t>((j % kStages) * geo.seg_bytes);
            const uint4* src = iss.src + c0 * 32 + lane;
            for (int c = 0; c < cnt; ++c) cp_async16(dst + c * 512u, src + c * 32);
        }
        cp_async_commit();  // empty groups keep the group count uniform
    };

    WarpTopK top;
    top.init(k);
    uint32_t issued = 0;
    for (; issued < kStages - 1; ++issued) issue(issued);
    // partial scores of a tile's parts, double-buffered by tile parity
    float* my_part = spart + gi * 2 * parts * 32;
    uint32_t j = 0;
    for (uint32_t i = 0; i < ntile_g; ++i) {
        float acc0 = 0.0f, acc1 = 0.0f;
        for (int jj = 0; jj < jmine; ++jj, ++j) {
            cp_async_wait<kStages - 2>();  // job j's group has landed (this lane's copies)
            const int g = j_lo + jj;
            const uint4* sbuf = reinterpret_cast<const uint4*>(ring + warp * kStages * geo.seg_bytes +
                                                               (j % kStages) * geo.seg_bytes);
            if (g < geo.ng)
                accumulate_blocks<BITS, GBL, GCH>(sbuf, lane, sq4, g * GBL, tb_addr, acc0, acc1);
            else
                accumulate_blocks<BITS, 8, TCH>(sbuf, lane, sq4, geo.ng * GBL, tb_addr, acc0, acc1);
            // job j's slot is free: this lane read its own entries above
            issue(issued++);
        }
        my_part[((i & 1) * parts + pi) * 32 + lane] = __fadd_rn(acc0, acc1);
        asm volatile("bar.sync %0, %1;" ::"r"(1 + gi), "r"(parts * 32) : "memory");
        if (pi == 0) {
            float S = my_part[((i & 1) * parts) * 32 + lane];
            for (int q = 1; q < parts; ++q) S = __fadd_rn(S, my_part[((i & 1) * parts + q) * 32 + lane]);
            const TileInfo cur = resolve(i);
            const size_t slot = static_cast<size_t>(cur.slot0) + lane;
            const bool valid = static_cast<uint32_t>(lane) < cur.nvalid;
            const float g1 = __ldg(ix.g1 + slot), h3 = __ldg(ix.h3 + slot);
            const float dist = __fmaf_rn(-__fmul_rn(2.0f, g1), S, __fadd_rn(cur.d2, h3));
            top.offer(dist, valid, [&] { return __ldg(ix.ids + slot); });
        }
    }
    cp_async_wait<0>();
    cta_merge(top, sm_d, sm_id, k);
    if (warp == 0) top.store(sw.part_d + static_cast<size_t>(blockIdx.x) * kMaxK,
                             sw.part_id + static_cast<size_t>(blockIdx.x) * kMaxK, k);
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(sw.counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // final merge: stage the per-CTA lists in shared memory (the ring is free
    // now) with coalesced loads, each warp folds a share into its own top-k
    // (batched bitonic merges), then one CTA merge
    top.init(k);
    const int Gi = static_cast<int>(gridDim.x);
    const int cap = (nw * kStages * geo.seg_bytes) / 8;
    float* st_d = reinterpret_cast<float*>(ring);
    uint32_t* st_i = reinterpret_cast<uint32_t*>(ring) + cap;
    const int total = Gi * k;
    for (int e0 = 0; e0 < total; e0 += cap) {
        const int m = min(cap, total - e0);
        __syncthreads();
        for (int e = tid; e < m; e += nt) {
            const int c = (e0 + e) / k, jj = (e0 + e) - c * k;
            st_d[e] = __ldcg(sw.part_d + static_cast<size_t>(c) * kMaxK + jj);
            st_i[e] = __ldcg(sw.part_id + static_cast<size_t>(c) * kMaxK + jj);
        }
        __syncthreads();
        for (int e = warp * 32; e < m; e += nw * 32) {
            const int i = e + lane;
            const bool okj = i < m;
            const float dd = okj ? st_d[i] : inf_f();
            const uint32_t ii = okj ? st_i[i] : 0xFFFFFFFFu;
            top.offer_pair(dd, ii, okj && ii != 0xFFFFFFFFu);
        }
    }
    cta_merge(top, sm_d, sm_id, k);
    if (warp == 0) top.store(out_d, out_ids, k);
    if (tid == 0) *sw.counter = 0;
}

template <int BITS>
int launch_bits(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k, const ScanWork& sw,
                const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s) {
    const size_t smem = scan_smem_bytes(ix, geo);
    // dynamic shared-memory opt-in, raised per device as needed
    static size_t configured[64] = {};
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    if (configured[dev & 63] < smem) {
        E8QC_CUDA(cudaFuncSetAttribute(scan_plain_kernel<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        configured[dev & 63] = smem;
    }
    scan_plain_kernel<BITS><<<sw.grid, geo.warps * 32, smem, s>>>(ix, rq, rw, nprobe, k, sw, geo, out_ids, out_d);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

}  // namespace

ScanGeo plain_scan_geo(const DevIndex& ix, size_t max_seg_bytes) {
    ScanGeo g{};
    const int gbl = group_blocks(ix.bits), gch = group_chunks(ix.bits);
    g.ng = ix.B / gbl;
    g.tail = (ix.B % gbl) != 0 ? 1 : 0;
    const int group_bytes = gch * 512;
    const int tch = (64 * ix.bits + 127) / 128;
    int U = static_cast<int>(max_seg_bytes / group_bytes);
    if (U < 1) U = 1;
    if (U > g.ng && g.ng > 0) U = g.ng;
    g.U = U;
    g.nseg = (g.ng + U - 1) / U + g.tail;
    int seg_chunks = U * gch;
    if (g.tail && tch > seg_chunks) seg_chunks = tch;
    g.seg_bytes = ((seg_chunks * 512) + 127) & ~127;
    // as many warps (a power of two <= 16) as the 227 KB shared-memory budget allows
    g.warps = kMaxWarps;
    while (g.warps > 2 && scan_smem_bytes(ix, g) > 225 * 1024) g.warps /= 2;  // powers of two
    return g;
}

size_t scan_smem_bytes(const DevIndex& ix, const ScanGeo& geo) {
    const int q = 1 << ix.bits;
    size_t b = static_cast<size_t>(geo.warps) * kStages * geo.seg_bytes;
    b += static_cast<size_t>(2) * q * table_rep(ix.bits) * 4;
    b += static_cast<size_t>(ix.pd) * 4;
    b += static_cast<size_t>(kToffCap + 1) * 4;
    b += static_cast<size_t>(geo.warps) * kMaxK * 8;
    b += static_cast<size_t>(2) * geo.warps * 32 * 4;
    b += 16;
    return b;
}

int launch_scan_plain(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k,
                      const ScanWork& sw, const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s) {
    switch (ix.bits) {
#define E8QC_CASE(b) \
    case b: return launch_bits<b>(ix, rq, rw, nprobe, k, sw, geo, out_ids, out_d, s);
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    return 0;
}

}  // namespace e8qc
