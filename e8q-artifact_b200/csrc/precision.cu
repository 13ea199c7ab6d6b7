// Precision search path: INT8 tensor-core candidate generation + exact
// rescoring.
//
// Every coordinate of a stored vector is one entry of a small level table
// (table[br][digit] = level / sqrt(Dpad), 2 x 2^bits values). The proxy of a
// coordinate is that entry quantised to int8 with one step for the whole
// table, p = rint(table / step), step = max|table| / 127 (an int8 lookup per
// digit, so each vector's proxy row is its level sequence to 8 bits). The
// query is quantised to int8 with a per-query scale qs, S8 = sum_i q8_i * p_i
// runs on tcgen05 kind::i8 with int32 accumulation in TMEM, and
//   S ~ S' = step * S8 / qs.
// The proxy distance D' = (d2 + h3) - 2*g1*S' of every (query, vector) pair
// is written, scaled per query, as fp16 to a scratch row per (query, list)
// pair in HBM (2 bytes per pair: far less than the codes the pair stands
// for); a per-query kernel then selects the query's best C proxies over all
// its rows, rescores those C candidates with the exact estimator of the plain
// scan (src/simd/e8q_search_generic.cpp:58-66; same table and per-block FMA
// chain, blocks summed in order into two alternating accumulators) and keeps
// the top-k. A rescored distance depends only on (query, vector), so results
// do not depend on what else is in the batch. An ME8Q index uses the same
// scan with each vector's coef-scaled levels quantised per vector
// (me8q_kernels.cu) and the ME8Q estimator for rescoring.
//
// The proxies of every vector are decoded once into an int8 "proxy plane"
// stored in the MMA operand layout (built on the first precision search), and
// the int8 query rows of a batch are gathered per (query, list) pair into the
// same layout, so the scan kernel moves both operands with 2D tensor-map (TMA)
// loads and does no decoding.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "decode_accum.cuh"
#include "device_common.cuh"
#include "internal.h"
#include "me8q.h"
#include "me8q_stream.cuh"
#include "precision.h"
#include "scan_plain.h"
#include "tc.cuh"
#include "tma.cuh"
#include "workspace.h"

namespace e8qc {

namespace {

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

constexpr int kPM = 128;  // pair rows per MMA tile (M = TMEM lanes)
constexpr int kPN = 256;  // vectors per MMA tile (N)
constexpr int kPK = 64;   // dimensions per staged K-chunk (2 MMAs of K = 32)
constexpr int kOrdCap = 512;  // final kernel: probes per query it orders nearest list first
constexpr size_t kFinalWideRows = 131072;  // select kernel: 4 warps per query from this many proxy rows
constexpr size_t kFinalWideBatch = 2048;   // ... and for batches below this size (too few queries to fill the GPU)

// Proxy candidates rescored per query, from the query's own k (so a query's
// result does not depend on the k of the others in its batch): the top
// max(32, 3k) by proxy distance, up to the 128 a warp's list holds. At k = 10
// the 32 already return the exact scan's top-10 (equal recall at every rate
// and nprobe measured); 40 (4k) pushes the select's per-warp lists past the
// 32-entry single-merge form and cost 0.15 ms per 4096-query batch.
__host__ __device__ constexpr int candidates_for(int k) {
    return (3 * k > 32 ? 3 * k : 32) < kMaxK ? (3 * k > 32 ? 3 * k : 32) : kMaxK;
}
constexpr size_t kScratchBudget = size_t(8) << 30;  // proxy rows per call chunk (bytes)

// Per-query int8 quantisation: q8 = rint(q * 127 / max|q|); per-query factor
// coef / qs and sum(q8).
__global__ void quantize_kernel(const float* __restrict__ rq, int pd, float coef, int with_sum,
                                int8_t* __restrict__ q8, float* __restrict__ qscale, float* __restrict__ qsum,
                                const float* __restrict__ pd2, const uint32_t* __restrict__ np_arr, int np_uniform,
                                int np_max, float* __restrict__ pscale) {
    __shared__ float red[32];
    __shared__ int ired[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const float* q = rq + static_cast<size_t>(blockIdx.x) * pd;
    float m = 0.0f;
    for (int i = tid; i < pd; i += blockDim.x) m = fmaxf(m, fabsf(q[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(kFull, m, o));
    if (lane == 0) red[warp] = m;
    __syncthreads();
    float amax = 0.0f;
    for (int i = 0; i < nw; ++i) amax = fmaxf(amax, red[i]);
    const float qs = amax > 0.0f ? 127.0f / amax : 1.0f;
    int sum = 0;
    for (int i = tid; i < pd; i += blockDim.x) {
        int v = __float2int_rn(q[i] * qs);
        v = v > 127 ? 127 : (v < -127 ? -127 : v);
        q8[static_cast<size_t>(blockIdx.x) * pd + i] = static_cast<int8_t>(v);
        sum += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
    if (lane == 0) ired[warp] = sum;
    __syncthreads();
    if (tid == 0) {
        int s = 0;
        for (int i = 0; i < nw; ++i) s += ired[i];
        qscale[blockIdx.x] = coef / qs;
        qsum[blockIdx.x] = with_sum ? static_cast<float>(s) : 0.0f;
        // proxy distances are stored as fp16 divided by the query's largest
        // routing distance (only their order within the query matters)
        const int np = np_arr ? static_cast<int>(np_arr[blockIdx.x]) : np_uniform;
        float dmax = 0.0f;
        for (int j = 0; j < np; ++j) dmax = fmaxf(dmax, pd2[static_cast<size_t>(blockIdx.x) * np_max + j]);
        pscale[blockIdx.x] = dmax > 0.0f ? 1.0f / dmax : 1.0f;
    }
}

// Start of each list's proxy rows: rowbase[L] = sum over lists L' < L of
// (pairs probing L') * stride(L'), stride = the list's padded slots (whole
// 32-vector tiles, so every row starts 128-byte aligned). One CTA of 1024
// threads.
__global__ void rowbase_kernel(const uint32_t* __restrict__ list_cnt, const uint32_t* __restrict__ tile_begin,
                               int nlist, unsigned long long* __restrict__ rowbase) {
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (int i0 = 0; i0 < nlist; i0 += blockDim.x) {
        const int i = i0 + tid;
        const unsigned long long v =
            i < nlist ? static_cast<unsigned long long>(list_cnt[i]) * ((tile_begin[i + 1] - tile_begin[i]) * 32ull)
                      : 0ull;
        unsigned long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long s = lane < nw ? wsum[lane] : 0ull;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(kFull, s, o);
                if (lane >= o) s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        if (i < nlist) rowbase[i] = carry + (warp > 0 ? wsum[warp - 1] : 0ull) + x - v;
        __syncthreads();
        if (tid == 0) carry += wsum[nw - 1];
        __syncthreads();
    }
}

// Proxies of one block (8 dims) as 8 packed int8: the quantised table entry
// of each digit (lut: 2 x 2^BITS int8, branch-major).
template <int BITS>
__device__ __forceinline__ uint2 block_proxy(const uint32_t* w, int base, const int8_t* __restrict__ lut) {
    uint32_t dg[8];
    const int br = decode_block<BITS>(w, base, dg);
    const int8_t* t = lut + (br ? (1 << BITS) : 0);
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t p = static_cast<uint32_t>(static_cast<uint8_t>(__ldg(t + dg[i])));
        if (i < 4) lo |= p << (8 * i);
        else hi |= p << (8 * (i - 4));
    }
    return make_uint2(lo, hi);
}

// Slot-major copy of the codes for the exact rescoring of scattered
// candidates: out[slot * nch + c] = chunk c of the slot (tile-major source:
// chunk c of lane l of tile t at codes[(t * nch + c) * 32 + l]). One thread
// per output chunk (coalesced writes).
__global__ void vcodes_kernel(const uint4* __restrict__ codes, size_t nslots, int nch, uint4* __restrict__ out) {
    const size_t total = nslots * static_cast<size_t>(nch);
    for (size_t e = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; e < total;
         e += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t slot = e / nch, c = e - slot * nch;
        out[e] = codes[((slot >> 5) * nch + c) * 32 + (slot & 31)];
    }
}

// Proxy plane: slot s, dimension i at byte (s/8)*8*pd + (i/16)*128 + (s%8)*16
// + i%16 -- 8-slot row groups of 16-byte core-matrix rows, the K-major
// no-swizzle operand layout of tcgen05, so the 64-dimension K-chunk kc of a
// row group is the 512 contiguous bytes at (s/8)*8*pd + kc*512. One thread per
// (slot, K-chunk): the slot's 2*BITS code words for those 64 dimensions,
// decoded into 64 proxies (four 16-byte stores; 8 consecutive slots fill 128
// contiguous bytes).
template <int BITS>
__global__ void __launch_bounds__(256) build_proxy_kernel(DevIndex ix, int nslots, const int8_t* __restrict__ lut,
                                                          unsigned char* __restrict__ plane) {
    constexpr int NW = 2 * BITS;
    const int slot = blockIdx.x * 256 + threadIdx.x;
    const int kc = blockIdx.y;
    if (slot >= nslots) return;
    const uint32_t* base =
        reinterpret_cast<const uint32_t*>(ix.codes + static_cast<size_t>(slot >> 5) * ix.nch * 32) + (slot & 31) * 4;
    uint32_t w[NW + 1];
#pragma unroll
    for (int j = 0; j < NW; j += 2) {
        const int wi = kc * NW + j;  // even: 8-byte aligned inside the lane's 16-byte entry
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(base + (wi >> 2) * 128 + (wi & 3)));
        w[j] = v.x;
        w[j + 1] = v.y;
    }
    w[NW] = 0u;
    uint32_t o[16];
#pragma unroll
    for (int blk = 0; blk < 8; ++blk) {
        const uint2 pr = block_proxy<BITS>(w, blk * 8 * BITS, lut);
        o[2 * blk] = pr.x;
        o[2 * blk + 1] = pr.y;
    }
    unsigned char* dst = plane + static_cast<size_t>(slot >> 3) * 8 * ix.pd + kc * 512 + (slot & 7) * 16;
#pragma unroll
    for (int c = 0; c < 4; ++c)
        *reinterpret_cast<uint4*>(dst + c * 128) = make_uint4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
}

// Query side of the MMA: the int8 query of every pair slot in the same row-
// group layout as the proxy plane (a list's pairs start at a multiple of 8, so
// a 128-pair work item is 16 whole row groups). Slots holding no pair, and the
// 128 rows past the end, are zero. Thread order: row within group fastest.
__global__ void gather_a8_kernel(const int8_t* __restrict__ q8, const uint32_t* __restrict__ pair_q, size_t pslots,
                                 size_t rows, int pd, unsigned char* __restrict__ a8) {
    const size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int nc = pd / 16;
    const size_t r8 = e & 7, rest = e >> 3;
    const size_t c = rest % nc, g = rest / nc;
    const size_t row = g * 8 + r8;
    if (row >= rows) return;
    const uint32_t qq = row < pslots ? pair_q[row] : 0xFFFFFFFFu;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (qq != 0xFFFFFFFFu) v = *reinterpret_cast<const uint4*>(q8 + static_cast<size_t>(qq) * pd + c * 16);
    *reinterpret_cast<uint4*>(a8 + g * 8 * pd + c * 128 + r8 * 16) = v;
}

// Persistent, warp-specialised proxy scan. Work items (one list, up to 128
// pair rows) come from a device queue; the producer takes them and publishes
// each through a 4-slot ring in shared memory (ifull / iempty mbarriers), so
// every role walks the same item -> 256-vector tile -> 64-dimension K-chunk
// sequence:
//   warp 0 (producer): per chunk, two 2D tensor-map (TMA) loads -- 16 query
//     row groups and 32 proxy row groups of 512 B (the chunk's 64 dimensions)
//     -- into a kStages ring, completing on full[s] (expect-tx);
//   warp 1 (one thread): waits full[s], issues the chunk's two kind::i8 MMAs
//     (M = 128 rows, N = 256 vectors, K = 32 each) into accumulator t % 2 of
//     two 256-column TMEM buffers, commits to empty[s]; after a tile's last
//     chunk commits to tfull[b];
//   warps 2..5 (epilogue): thread r of warp w owns pair row 32*(w%4) + lane
//     (the TMEM lane quarter the warp may read). Per tile the warp stages the
//     tile's (-2*g1, h3) in its own shared table (prefetched one tile ahead
//     within an item), reads its row of the accumulator 32 columns at a time,
//     writes its row's 32 proxy distances as eight 16-byte stores, then
//     arrives on tempty[b].
// Every wait is bounded; a timeout sets a CTA-wide abort flag that ends all
// roles' loops, is reported through the error word, and the CTA frees its TMEM
// after its outstanding copies and MMAs have completed (or a last bounded wait
// for them ran out). No role waits on a barrier that another role can skip.
constexpr int kScanThreads = 192;
constexpr uint32_t kScanCols = 512;
constexpr int kStageBytes = kPM * kPK + kPN * kPK;  // 8 KB queries + 16 KB proxies
constexpr int kRing = 4;                            // items in flight between roles

template <int kStages>
__global__ void __launch_bounds__(kScanThreads, 1) precision_scan_kernel(
    DevIndex ix, const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
    const uint32_t* __restrict__ pair_q,
    const float* __restrict__ pair_d2, const float* __restrict__ qscale, const float* __restrict__ qsum,
    const uint4* __restrict__ items, const uint32_t* __restrict__ n_items, uint32_t* __restrict__ head,
    const uint32_t* __restrict__ pair_off, const unsigned long long* __restrict__ rowbase, __half* __restrict__ prox,
    const float* __restrict__ pscale, unsigned long long* __restrict__ counts, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char psm[];
    float2* ghtab = reinterpret_cast<float2*>(psm + kStages * kStageBytes);  // 4 warps x kPN
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], tfull[2], tempty[2], ifull[kRing],
        iempty[kRing], fin;
    __shared__ uint4 s_items[kRing];
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int pd = ix.pd, nK = pd / kPK;
    if (warp == 0) {
        tc::tmem_alloc(&s_tmem, kScanCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < kStages; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < kRing; ++i) {
            mbar_init(&ifull[i], 1);
            mbar_init(&iempty[i], 5);  // the MMA thread + one lane per epilogue warp
        }
        mbar_init(&tfull[0], 1);
        mbar_init(&tfull[1], 1);
        mbar_init(&tempty[0], 4);
        mbar_init(&tempty[1], 4);
        mbar_init(&fin, 1);
        s_abort = 0;
        fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = s_tmem;
    const uint32_t NI = *n_items;

    if (warp == 0) {
        // ---- producer ----
        uint32_t f = 0;  // chunk fills issued
        for (uint32_t n = 0; !s_abort; ++n) {
            const uint32_t j = n % kRing;
            if (n >= kRing && !mbar_wait_or_abort(&iempty[j], ((n / kRing) - 1) & 1u, &s_abort)) break;
            if (lane == 0) {
                const uint32_t it = atomicAdd(head, 1u);
                s_items[j] = it < NI ? items[it] : make_uint4(0xFFFFFFFFu, 0, 0, 0);
                mbar_arrive(&ifull[j]);
            }
            __syncwarp();
            const uint4 item = s_items[j];
            if (item.x == 0xFFFFFFFFu) break;
            const uint32_t L = item.x, pbase = item.y;
            const uint32_t len = ix.list_len[L], tile0 = ix.tile_begin[L];
            const int arow = static_cast<int>(pbase >> 3);  // the item's first query row group
            for (uint32_t v0 = 0; v0 < len && !s_abort; v0 += kPN) {
                const int brow = static_cast<int>((tile0 * 32u + v0) >> 3);  // the tile's first proxy row group
                for (int kc = 0; kc < nK; ++kc, ++f) {
                    const int st = static_cast<int>(f % kStages);
                    if (f >= static_cast<uint32_t>(kStages) &&
                        !mbar_wait_or_abort(&empty[st], ((f / kStages) - 1) & 1u, &s_abort))
                        break;
                    if (lane == 0) {
                        unsigned char* sA = psm + st * kStageBytes;
                        unsigned char* sB = sA + kPM * kPK;
                        mbar_arrive_expect_tx(&full[st], kStageBytes);
                        // boxes of 32 (B) and 16 (A) row groups x 512 bytes (128 u32 at x = kc * 128)
                        tma_load_2d(sB, &map_b, kc * 128, brow, &full[st]);
                        tma_load_2d(sA, &map_a, kc * 128, arow, &full[st]);
                    }
                    __syncwarp();
                }
            }
        }
        // copies still in flight land before the CTA can exit
        if (s_abort && lane == 0)
            for (uint32_t g = f > kStages ? f - kStages : 0; g < f; ++g)
                (void)mbar_wait_bounded(&full[g % kStages], (g / kStages) & 1u, 100u);
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_i8(kPM, kPN);
            const uint32_t sbo = (kPK / 16) * 128u;
            uint32_t c = 0, t = 0;
            bool issued = false;
            for (uint32_t n = 0; !s_abort; ++n) {
                const uint32_t j = n % kRing;
                if (!mbar_wait_or_abort(&ifull[j], (n / kRing) & 1u, &s_abort)) break;
                const uint4 item = s_items[j];
                if (item.x == 0xFFFFFFFFu) break;
                const uint32_t len = ix.list_len[item.x];
                for (uint32_t v0 = 0; v0 < len && !s_abort; v0 += kPN, ++t) {
                    const uint32_t b = t & 1u;
                    if (t >= 2 && !mbar_wait_or_abort(&tempty[b], ((t >> 1) - 1) & 1u, &s_abort)) break;
                    tc::fence_after_sync();
                    const uint32_t d_tmem = tmem + b * 256u;
                    for (int kc = 0; kc < nK; ++kc, ++c) {
                        const int st = static_cast<int>(c % kStages);
                        if (!mbar_wait_or_abort(&full[st], (c / kStages) & 1u, &s_abort)) break;
                        tc::fence_after_sync();
                        const uint32_t a0 = tc::saddr(psm + st * kStageBytes), b0 = a0 + kPM * kPK;
#pragma unroll
                        for (int s2 = 0; s2 < kPK / 32; ++s2)
                            tc::mma_i8(d_tmem, tc::smem_desc(a0 + 256u * s2, 128u, sbo),
                                       tc::smem_desc(b0 + 256u * s2, 128u, sbo), idesc, (kc > 0 || s2 > 0) ? 1u : 0u);
                        tc::mma_commit(&empty[st]);
                        issued = true;
                    }
                    if (s_abort) break;
                    tc::mma_commit(&tfull[b]);
                }
                mbar_arrive(&iempty[j]);
            }
            // every MMA issued has completed before TMEM is released
            if (issued) {
                tc::mma_commit(&fin);
                (void)mbar_wait_bounded(&fin, 0u, 200u);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue ----
        const int q4 = warp & 3;  // TMEM lane quarter this warp may read
        const int r = q4 * 32 + lane;
        float2* gh = ghtab + (warp - 2) * kPN;
        uint32_t t = 0;
        for (uint32_t n = 0; !s_abort; ++n) {
            const uint32_t j = n % kRing;
            if (!mbar_wait_or_abort(&ifull[j], (n / kRing) & 1u, &s_abort)) break;
            const uint4 item = s_items[j];
            if (item.x == 0xFFFFFFFFu) break;
            const uint32_t L = item.x, pbase = item.y;
            const int m = static_cast<int>(item.z);
            const uint32_t len = ix.list_len[L], tile0 = ix.tile_begin[L];
            const uint32_t stride = (ix.tile_begin[L + 1] - tile0) * 32u;
            float sc = 0.0f, sum = 0.0f, d2 = 0.0f, ps = 1.0f;
            __half* row = prox;
            if (r < m) {
                const uint32_t qq = pair_q[pbase + r];
                sc = qscale[qq];
                sum = qsum[qq];
                ps = pscale[qq];
                d2 = pair_d2[pbase + r];
                row = prox + rowbase[L] + static_cast<unsigned long long>(pbase + r - pair_off[L]) * stride;
            }
            if (warp == 2 && lane == 0) {
                atomicAdd(counts, static_cast<unsigned long long>(len) * m);  // (query, vector) pairs
                atomicAdd(counts + 1, static_cast<unsigned long long>(len));  // vectors read
                if (item.w == 0) atomicAdd(counts + 2, static_cast<unsigned long long>(len));  // once per list
            }
            // (g1, h3) of columns 4*lane.. and 128 + 4*lane.. of a tile (zero past the padded list)
            const float4* g4 = reinterpret_cast<const float4*>(ix.g1 + tile0 * 32u);
            const float4* h4 = reinterpret_cast<const float4*>(ix.h3 + tile0 * 32u);
            float4 ga = make_float4(0.f, 0.f, 0.f, 0.f), gb = ga, ha = ga, hb = ga;
            auto fetch = [&](uint32_t v0) {
                const uint32_t ca = v0 + 4 * lane, cb = ca + 128;
                ga = ca < stride ? __ldg(g4 + (ca >> 2)) : make_float4(0.f, 0.f, 0.f, 0.f);
                ha = ca < stride ? __ldg(h4 + (ca >> 2)) : make_float4(0.f, 0.f, 0.f, 0.f);
                gb = cb < stride ? __ldg(g4 + (cb >> 2)) : make_float4(0.f, 0.f, 0.f, 0.f);
                hb = cb < stride ? __ldg(h4 + (cb >> 2)) : make_float4(0.f, 0.f, 0.f, 0.f);
            };
            fetch(0);
            for (uint32_t v0 = 0; v0 < len; v0 += kPN, ++t) {
                const uint32_t b = t & 1u;
                __syncwarp();  // every lane is done reading the previous tile's table
                gh[4 * lane + 0] = make_float2(-__fmul_rn(2.0f, ga.x), ha.x);
                gh[4 * lane + 1] = make_float2(-__fmul_rn(2.0f, ga.y), ha.y);
                gh[4 * lane + 2] = make_float2(-__fmul_rn(2.0f, ga.z), ha.z);
                gh[4 * lane + 3] = make_float2(-__fmul_rn(2.0f, ga.w), ha.w);
                gh[128 + 4 * lane + 0] = make_float2(-__fmul_rn(2.0f, gb.x), hb.x);
                gh[128 + 4 * lane + 1] = make_float2(-__fmul_rn(2.0f, gb.y), hb.y);
                gh[128 + 4 * lane + 2] = make_float2(-__fmul_rn(2.0f, gb.z), hb.z);
                gh[128 + 4 * lane + 3] = make_float2(-__fmul_rn(2.0f, gb.w), hb.w);
                __syncwarp();
                if (v0 + kPN < len) fetch(v0 + kPN);  // next tile of this item, in flight meanwhile
                if (!mbar_wait_or_abort(&tfull[b], (t >> 1) & 1u, &s_abort)) break;
                tc::fence_after_sync();
                for (uint32_t c0 = 0; c0 < static_cast<uint32_t>(kPN) && v0 + c0 < len; c0 += 32) {
                    uint32_t acc[32];
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj) {
                        uint32_t(&part)[8] = *reinterpret_cast<uint32_t(*)[8]>(acc + 8 * jj);
                        tc::tmem_ld8(tmem + ((static_cast<uint32_t>(q4) * 32u) << 16) + b * 256u + c0 + 8 * jj,
                                     part);
                    }
                    tc::tmem_ld_wait();
                    if (r < m) {
                        // columns past len land in the row's tile padding (rows are whole tiles)
                        uint4* dst = reinterpret_cast<uint4*>(row + v0 + c0);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            uint32_t hw[4];
#pragma unroll
                            for (int e2 = 0; e2 < 4; ++e2) {
                                float o[2];
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                    const int e = 8 * q + 2 * e2 + h;
                                    const float2 cg = gh[c0 + e];
                                    const float Sp =
                                        sc * __fmaf_rn(2.0f, static_cast<float>(static_cast<int>(acc[e])), sum);
                                    o[h] = __fmul_rn(__fmaf_rn(cg.x, Sp, __fadd_rn(d2, cg.y)), ps);
                                }
                                const __half2 hv = __floats2half2_rn(o[0], o[1]);
                                hw[e2] = *reinterpret_cast<const uint32_t*>(&hv);
                            }
                            dst[q] = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                        }
                    }
                }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[b]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&iempty[j]);
        }
    }
    __syncthreads();
    if (s_abort && tid == 0) atomicOr(err, kErrWaitTimeout);
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, kScanCols);
}

// Exact ME8Q estimate of stored slot `slot` for a rotated query q (shared
// memory) whose routing distance to the slot's list is d2, in the
// reference's form (EstimateRow, src/index/me8q_search.cpp:74-95): per coded
// run an fp32 score S_s = sum q * level accumulated in dimension order, then
// d2 + sum_s (h2_s - 2 coef_s S_s) in fp64 (h2_s alone when coef_s is 0).
__device__ float me8q_rescore(const Me8qView& mv, uint32_t slot, const float* q, float d2) {
    double acc = static_cast<double>(d2);
    const int nch = mv.base.nch;
    for (int r = 0; r < mv.nruns; ++r) {
        const Me8qRun run = mv.runs[r];
        if (run.bits == 0) continue;
        const double cf = static_cast<double>(__ldg(mv.coef + static_cast<size_t>(run.coded) * mv.nslots + slot));
        const double hh = static_cast<double>(__ldg(mv.h2 + static_cast<size_t>(run.coded) * mv.nslots + slot));
        if (cf == 0.0) {
            acc += hh;
            continue;
        }
        const float* lev0 = mv.levels + mv.chunks[run.off / 64].lev;
        const int qb = 1 << run.bits;
        float sc = 0.0f;
        for (int j = 0; j < run.len / 8; ++j) {
            uint32_t dg[8];
            const int br = me8q_block(mv.base.codes, nch, slot, run.word0, run.bits, j, dg);
            const float* lv = lev0 + (br ? qb : 0);
#pragma unroll
            for (int i = 0; i < 8; ++i) sc = __fmaf_rn(q[run.off + j * 8 + i], __ldg(lv + dg[i]), sc);
        }
        acc += __fma_rn(-2.0 * cf, static_cast<double>(sc), hh);
    }
    return static_cast<float>(acc);
}

constexpr uint32_t kHalfInf2 = 0x7C007C00u;  // two fp16 +inf
__device__ __forceinline__ __half2 u32_as_half2(uint32_t w) { return *reinterpret_cast<const __half2*>(&w); }

// Per query (FW warps of a 4-warp block; 4/FW queries per block): the best
// C proxies over the query's rows, written as candidate slots for the
// rescoring kernel. FW = 4 for queries with many rows (long per-query
// chains), 1 otherwise.
//
// Rows are visited nearest list first (routing distance, then probe index):
// the best proxies mostly sit in the nearest lists, so the thresholds settle
// on the first rows and later steps pass the filter without offers (a query
// with more than kOrdCap probes keeps list order). Warp w of a query streams
// the rows of probes w, w + FW, ... keeping its own top-C; the query's warps
// publish their C-th best in shared memory and each filters with the
// smallest of them (a value above another warp's C-th best has C better
// values and cannot be in the query's top C). The query's first warp merges
// the FW lists. The kernel holds no level table or query, so many warps stay
// resident to keep the row reads in flight.
template <int FW>
__global__ void __launch_bounds__(128, 8) precision_select_kernel(
    DevIndex ix, const __half* __restrict__ prox, const unsigned long long* __restrict__ rowbase,
    const uint32_t* __restrict__ pair_off, const uint32_t* __restrict__ pos_of, const uint32_t* __restrict__ probes,
    const float* __restrict__ pd2, int nq, const uint32_t* __restrict__ np_arr, int np_max,
    const uint32_t* __restrict__ k_arr, int k_uniform, uint32_t* __restrict__ cand_out) {
    static_assert(FW == 1 || FW == 2 || FW == 4, "warps per query");
    constexpr int QPB = 4 / FW;  // queries per block
    __shared__ __align__(16) float sbufs[4 * 512];        // per warp: one step of values; the query's d2 staging
    __shared__ float cd[(FW > 1 ? 4 : 1) * kMaxK];      // per warp: candidate proxies (merge of FW lists)
    __shared__ uint32_t ci[(FW > 1 ? 4 : 1) * kMaxK];   // per warp: candidate slots
    __shared__ uint16_t ords[QPB * kOrdCap];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int qi = warp / FW, wq = warp % FW;  // query slot in the block, warp within the query
    uint16_t* ord = ords + qi * kOrdCap;
    __shared__ float s_thr[4];
    const int q = blockIdx.x * QPB + qi;
    const bool qvalid = q < nq;
    const int np = qvalid ? (np_arr ? static_cast<int>(np_arr[q]) : np_max) : 0;
    const int kq = qvalid ? (k_arr ? static_cast<int>(k_arr[q]) : k_uniform) : 0;
    const int C = candidates_for(kq);  // the query's own candidate count (uniform within the query's warps)
    const uint32_t* pr = probes + static_cast<size_t>(qvalid ? q : 0) * np_max;
    const bool reorder = np <= kOrdCap;
    float* qstage = sbufs + qi * FW * 512;  // FW*512 >= kOrdCap floats: the query's d2 staging
    if (reorder)
        for (int i = wq * 32 + lane; i < np; i += FW * 32) qstage[i] = pd2[static_cast<size_t>(q) * np_max + i];
    __syncthreads();
    if (reorder)
        for (int i = wq * 32 + lane; i < np; i += FW * 32) {
            const float di = qstage[i];
            int r = 0;
            for (int j = 0; j < np; ++j) {
                const float dj = qstage[j];
                r += (dj < di) | ((dj == di) & (j < i));
            }
            ord[r] = static_cast<uint16_t>(i);
        }
    if (tid < 4) s_thr[tid] = inf_f();
    __syncthreads();
    volatile float* vthr = s_thr + qi * FW;
    float* sbuf = sbufs + warp * 512;

    // 1. best C proxies of this warp's rows (slot as tie-break). Row metadata
    //    for 32 of the warp's probes at a time sits in registers (lane j: the
    //    warp's probe w0 + j) and is read by shuffle; values stream 512 per
    //    step, two steps in flight ahead of the one being filtered.
    const int npw = np > wq ? (np - wq + FW - 1) / FW : 0;
    WarpTopK cand;
    cand.init(C);
    int w0 = -32;
    unsigned long long m_off = 0;  // this lane's row: element offset into prox
    uint32_t m_len = 0, m_slot0 = 0;
    auto load_window = [&](int base) {
        w0 = base;
        const int i = base + lane;
        m_off = 0;
        m_len = 0;
        m_slot0 = 0;
        if (i < npw) {
            const int p = wq + FW * i;
            const int pp = reorder ? static_cast<int>(ord[p]) : p;
            const uint32_t L = pr[pp];
            const uint32_t t0 = ix.tile_begin[L];
            const uint32_t stride = (ix.tile_begin[L + 1] - t0) * 32u;
            const uint32_t pos = pos_of[static_cast<size_t>(q) * np_max + pp];
            m_off = rowbase[L] + static_cast<unsigned long long>(pos - pair_off[L]) * stride;
            m_len = ix.list_len[L];
            m_slot0 = t0 * 32u;
        }
    };
    struct Step {
        int p;
        uint32_t v0, len, slot0;
        unsigned long long off;
    };
    // the step after (p, v0 + 512), skipping empty rows; p >= npw when done
    auto advance = [&](int p, uint32_t v0, uint32_t len) {
        Step st{p, v0 + 512, len, 0, 0};
        if (st.v0 >= len) {
            st.p = p + 1;
            st.v0 = 0;
            for (;; ++st.p) {
                if (st.p >= npw) break;
                if (st.p >= w0 + 32) load_window(w0 + 32);
                const uint32_t l = __shfl_sync(kFull, m_len, st.p - w0);
                if (l > 0) break;
            }
        }
        if (st.p < npw) {
            st.len = __shfl_sync(kFull, m_len, st.p - w0);
            st.slot0 = __shfl_sync(kFull, m_slot0, st.p - w0);
            st.off = __shfl_sync(kFull, m_off, st.p - w0);
        }
        return st;
    };
    // a step: 512 fp16 values of the row, lane l holding columns 8l..8l+7 and
    // 256+8l..256+8l+7 (one 16-byte load each)
    auto load_step = [&](const Step& st, uint4 (&x)[2]) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint32_t va = st.v0 + 256 * j + 8 * lane;
            x[j] = (st.p < npw && va < st.len) ? __ldcs(reinterpret_cast<const uint4*>(prox + st.off) + (va >> 3))
                                               : make_uint4(kHalfInf2, kHalfInf2, kHalfInf2, kHalfInf2);
        }
    };
    load_window(0);
    Step cur = advance(-1, 0, 0);  // first non-empty row
    uint4 cx[2];
    load_step(cur, cx);
    Step nxt = advance(cur.p, cur.v0, cur.len);
    uint4 nx[2];
    load_step(nxt, nx);
    while (cur.p < npw) {
        const Step nn = advance(nxt.p, nxt.v0, nxt.len);
        uint4 nnx[2];
        load_step(nn, nnx);
        // filter: a 16-bit mask per lane of the values that can enter the
        // query's top C; value t of this lane is column 256*(t/8) + 8*lane + t%8
        float filt = cand.thr_d;
        if constexpr (FW > 1) {
#pragma unroll
            for (int w2 = 0; w2 < FW; ++w2) filt = fminf(filt, vthr[w2]);
        }
        // quick test first: can any of the lane's 16 values pass? (for a half
        // v and a float f, v > f exactly when v > f rounded down to a half)
        __half2 mn = __hmin2(__hmin2(__hmin2(u32_as_half2(cx[0].x), u32_as_half2(cx[0].y)),
                                     __hmin2(u32_as_half2(cx[0].z), u32_as_half2(cx[0].w))),
                             __hmin2(__hmin2(u32_as_half2(cx[1].x), u32_as_half2(cx[1].y)),
                                     __hmin2(u32_as_half2(cx[1].z), u32_as_half2(cx[1].w))));
        const bool maybe = __hle2_mask(mn, __half2half2(__float2half_rd(filt))) != 0u;
        if (!__any_sync(kFull, maybe)) {
            cur = nxt;
            cx[0] = nx[0];
            cx[1] = nx[1];
            nxt = nn;
            nx[0] = nnx[0];
            nx[1] = nnx[1];
            continue;
        }
        float v[16];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const uint32_t w4[4] = {cx[j].x, cx[j].y, cx[j].z, cx[j].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w4[e]));
                v[8 * j + 2 * e] = f.x;
                v[8 * j + 2 * e + 1] = f.y;
            }
        }
        uint32_t hit = 0;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            const uint32_t va = cur.v0 + 256 * (t >> 3) + 8 * lane + (t & 7);
            hit |= static_cast<uint32_t>(va < cur.len && !(v[t] > filt)) << t;
        }
        if (__any_sync(kFull, hit != 0)) {
            // staged in shared memory so the offer loop indexes it
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                float4* dst = reinterpret_cast<float4*>(sbuf + 256 * j + 8 * lane);
                dst[0] = make_float4(v[8 * j + 0], v[8 * j + 1], v[8 * j + 2], v[8 * j + 3]);
                dst[1] = make_float4(v[8 * j + 4], v[8 * j + 5], v[8 * j + 6], v[8 * j + 7]);
            }
            __syncwarp();
            // one offer per round: each lane its lowest remaining hit; offer()
            // re-checks every value against the warp's threshold of that moment
#pragma unroll 1
            while (__any_sync(kFull, hit != 0)) {
                const bool has = hit != 0;
                const int t = has ? __ffs(static_cast<int>(hit)) - 1 : 0;
                hit &= hit - 1u;
                const uint32_t col = 256u * static_cast<uint32_t>(t >> 3) + 8u * static_cast<uint32_t>(lane) +
                                     static_cast<uint32_t>(t & 7);
                cand.offer_pair(has ? sbuf[col] : inf_f(), cur.slot0 + cur.v0 + col, has);
            }
            __syncwarp();
            if constexpr (FW > 1)
                if (lane == 0) vthr[wq] = cand.thr_d;
        }
        cur = nxt;
        cx[0] = nx[0];
        cx[1] = nx[1];
        nxt = nn;
        nx[0] = nnx[0];
        nx[1] = nnx[1];
    }
    // 2. the query's first warp merges its warps' lists into the query's top C
    //    and writes the candidate slots (C of them, padding UINT32_MAX)
    if constexpr (FW > 1) {
        const float* qcd = cd + qi * FW * kMaxK;
        const uint32_t* qci = ci + qi * FW * kMaxK;
        cand.store(cd + warp * kMaxK, ci + warp * kMaxK, C);
        __syncthreads();
        if (wq == 0) {
            for (int w2 = 1; w2 < FW; ++w2)
                for (int s2 = 0; s2 * 32 < C; ++s2) {
                    const int j = s2 * 32 + lane;
                    const bool in = j < C && qci[w2 * kMaxK + j] != 0xFFFFFFFFu;
                    cand.offer_pair(in ? qcd[w2 * kMaxK + j] : inf_f(), in ? qci[w2 * kMaxK + j] : 0xFFFFFFFFu, in);
                }
        }
    }
    if (wq == 0 && qvalid) {
#pragma unroll
        for (int s2 = 0; s2 < 4; ++s2) {
            const int j = s2 * 32 + lane;
            if (j < C) cand_out[static_cast<size_t>(q) * kMaxK + j] = cand.id[s2];
        }
    }
}

// Routing distance of (query, the list holding `slot`): the query's probes
// (np of them, in list order) are binary-searched for the slot's list.
__device__ __forceinline__ float rescore_d2(const DevIndex& ix, const uint32_t* __restrict__ pr, int np,
                                            const float* __restrict__ qpd2, uint32_t slot) {
    const uint32_t list = __ldg(ix.list_of_tile + (slot >> 5));
    int lo = 0, hi = np;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pr[mid] <= list) lo = mid;
        else hi = mid;
    }
    return qpd2[lo];
}

// Exact rescoring of each query's C candidates (E8Q estimator at BITS, or
// the ME8Q estimator) and the top k by exact distance. Four queries per
// 4-warp block; the (query, 32-candidate chunk) units of the block are dealt
// over its warps, then warp w keeps the top k of query w.
template <int BITS, bool ME8Q, int QPB>
__global__ void __launch_bounds__(128) precision_rescore_kernel(
    DevIndex ix, Me8qView mv, const float* __restrict__ rq, const uint32_t* __restrict__ cand,
    const uint32_t* __restrict__ probes, const float* __restrict__ pd2, int nq, const uint32_t* __restrict__ np_arr,
    int np_max, const uint32_t* __restrict__ k_arr, int k_uniform, int out_stride, uint32_t* __restrict__ out_ids,
    float* __restrict__ out_d) {
    constexpr int Q = 1 << BITS;
    constexpr int REP = table_rep(BITS);
    constexpr int GBL = group_blocks(BITS), GCH = group_chunks(BITS);
    constexpr int TCH = (64 * BITS + 127) / 128;
    extern __shared__ __align__(16) float fsm[];
    const int pd = ix.pd;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float* tabrep = fsm;                                        // 2*Q*REP (E8Q)
    float* myqs = tabrep + (ME8Q ? 0 : 2 * Q * REP);              // QPB rotated queries
    float* cd = myqs + QPB * pd;                                  // QPB queries x kMaxK exact distances
    uint32_t* ci = reinterpret_cast<uint32_t*>(cd + QPB * kMaxK);  // QPB queries x kMaxK slots, then ids
    const int q0 = blockIdx.x * QPB;
    if constexpr (!ME8Q)
        for (int e = tid; e < 2 * Q * REP; e += blockDim.x) tabrep[e] = ix.tab[e / REP];
    int nunit[QPB], Cq[QPB];
#pragma unroll
    for (int t = 0; t < QPB; ++t) {
        const int q = q0 + t;
        Cq[t] = q < nq ? candidates_for(k_arr ? static_cast<int>(k_arr[q]) : k_uniform) : 0;
        nunit[t] = (Cq[t] + 31) / 32;
    }
    for (int e = tid; e < QPB * pd; e += blockDim.x) {
        const int t = e / pd, i = e - t * pd;
        myqs[e] = q0 + t < nq ? rq[static_cast<size_t>(q0 + t) * pd + i] : 0.0f;
    }
    for (int e = tid; e < QPB * kMaxK; e += blockDim.x) {
        const int t = e / kMaxK, j = e - t * kMaxK;
        ci[e] = j < Cq[t] ? cand[static_cast<size_t>(q0 + t) * kMaxK + j] : 0xFFFFFFFFu;
    }
    __syncthreads();
    // 3. exact rescoring: unit u = (query t, candidates 32c..32c+31); each lane
    //    writes its candidate's (distance, id) over its slot entry
    int total = 0;
#pragma unroll
    for (int t = 0; t < QPB; ++t) total += nunit[t];
    for (int u = warp; u < total; u += 4) {
        int t = 0, c = u;
        while (c >= nunit[t]) c -= nunit[t++];
        const int q = q0 + t;
        const int np = np_arr ? static_cast<int>(np_arr[q]) : np_max;
        const uint32_t* pr = probes + static_cast<size_t>(q) * np_max;
        const float* myq = myqs + t * pd;
        const int j = c * 32 + lane;
        const uint32_t slot = j < Cq[t] ? ci[t * kMaxK + j] : 0xFFFFFFFFu;
        const bool live = slot != 0xFFFFFFFFu;
        float dist = inf_f();
        uint32_t gid = 0xFFFFFFFFu;
        if constexpr (ME8Q) {
            if (live) {
                const float d2 = rescore_d2(ix, pr, np, pd2 + static_cast<size_t>(q) * np_max, slot);
                dist = me8q_rescore(mv, slot, myq, d2);
            }
        } else if (live) {
            // The candidate's codes (slot-major copy, contiguous) stream
            // through a ring of PF prefetched groups; the factors and id are
            // loaded and the routing distance searched while they are in flight.
            constexpr int PF = GCH >= 12 ? 1 : (12 / GCH >= 3 ? 3 : 12 / GCH);
            const uint4* vp = ix.vcodes + static_cast<size_t>(slot) * ix.nch;
            const int ng = (pd / 8) / GBL;
            const bool tail = ((pd / 8) % GBL) != 0;
            uint4 ring[PF][GCH];
#pragma unroll
            for (int r = 0; r < PF; ++r)
                if (r < ng)
#pragma unroll
                    for (int c = 0; c < GCH; ++c) ring[r][c] = __ldg(vp + r * GCH + c);
            const float g1 = __ldg(ix.g1 + slot), h3 = __ldg(ix.h3 + slot);
            gid = __ldg(ix.ids + slot);
            const float d2 = rescore_d2(ix, pr, np, pd2 + static_cast<size_t>(q) * np_max, slot);
            const uint32_t tb_addr = static_cast<uint32_t>(__cvta_generic_to_shared(tabrep)) + (lane % REP) * 4u;
            const float4* sq4 = reinterpret_cast<const float4*>(myq);
            float acc0 = 0.0f, acc1 = 0.0f;
            for (int g = 0; g < ng; ++g) {
                uint4 cur[GCH];
#pragma unroll
                for (int c = 0; c < GCH; ++c) cur[c] = ring[0][c];
#pragma unroll
                for (int r = 0; r + 1 < PF; ++r)
#pragma unroll
                    for (int c = 0; c < GCH; ++c) ring[r][c] = ring[r + 1][c];
                if (g + PF < ng)
#pragma unroll
                    for (int c = 0; c < GCH; ++c) ring[PF - 1][c] = __ldg(vp + (g + PF) * GCH + c);
                accumulate_regs<BITS, GBL, GCH>(cur, sq4, g * GBL, tb_addr, acc0, acc1);
            }
            if (tail) accumulate_blocks<BITS, 8, TCH, 1>(vp + ng * GCH, 0, sq4, ng * GBL, tb_addr, acc0, acc1);
            const float S = __fadd_rn(acc0, acc1);
            dist = __fmaf_rn(-__fmul_rn(2.0f, g1), S, __fadd_rn(d2, h3));
        }
        if (live && ME8Q) gid = __ldg(ix.ids + slot);
        if (j < Cq[t]) {
            cd[t * kMaxK + j] = dist;
            ci[t * kMaxK + j] = gid;
        }
    }
    __syncthreads();
    // 4. top k by exact distance: warp w < QPB, query q0 + w
    const int q = q0 + warp;
    if (warp < QPB && q < nq) {
        const int kq = k_arr ? static_cast<int>(k_arr[q]) : k_uniform;
        int C = 0;
#pragma unroll
        for (int t = 0; t < QPB; ++t)
            if (t == warp) C = Cq[t];
        const float* qcd = cd + warp * kMaxK;
        const uint32_t* qci = ci + warp * kMaxK;
        WarpTopK top;
        top.init(kq);
        for (int s2 = 0; s2 * 32 < C; ++s2) {
            const int j = s2 * 32 + lane;
            const bool in = j < C && qci[j] != 0xFFFFFFFFu;
            top.offer_pair(in ? qcd[j] : inf_f(), in ? qci[j] : 0xFFFFFFFFu, in);
        }
#pragma unroll
        for (int s3 = 0; s3 < 4; ++s3) {
            const int j = s3 * 32 + lane;
            if (j < out_stride) {
                const bool in = j < kq;
                out_d[static_cast<size_t>(q) * out_stride + j] = in ? top.d[s3] : inf_f();
                out_ids[static_cast<size_t>(q) * out_stride + j] = in ? top.id[s3] : 0xFFFFFFFFu;
            }
        }
    }
}

constexpr size_t scan_smem(int stages) {
    return static_cast<size_t>(stages) * kStageBytes + static_cast<size_t>(4) * kPN * 8;
}

}  // namespace

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        E8QC_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) fail(E8QC_ECUDA, "cuTensorMapEncodeTiled is unavailable");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// A row-group plane (rows of 8 * pd bytes, seen as 2 * pd u32) as a 2D tensor
// map whose box is box_rows row groups x box_u32 u32 (512 bytes: one 64-byte
// K-chunk of each of the 8 rows).
CUtensorMap plane_map(const void* base, size_t row_groups, int pd, uint32_t box_rows, uint32_t box_u32) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(2 * pd), static_cast<cuuint64_t>(row_groups)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(8) * pd};
    const cuuint32_t box[2] = {box_u32, box_rows};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = encode_tiled()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<void*>(base), dims, strides,
                                      box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(E8QC_ECUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

namespace {

template <int STAGES>
void launch_scan_stages(const DevIndex& ix, Workspace& ws, const CUtensorMap& map_a, const CUtensorMap& map_b,
                        cudaStream_t s) {
    int dev = 0, sms = 148;
    E8QC_CUDA(cudaGetDevice(&dev));
    constexpr size_t smem = scan_smem(STAGES);
    static bool configured[64] = {};
    if (!configured[dev & 63]) {
        E8QC_CUDA(cudaFuncSetAttribute(precision_scan_kernel<STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        configured[dev & 63] = true;
    }
    E8QC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint32_t* nitems = ws.b_nitems.as<uint32_t>();
    ws.mark_scan(false, s);
    // one CTA per SM: the two accumulators take all 512 TMEM columns
    precision_scan_kernel<STAGES><<<sms, kScanThreads, smem, s>>>(
        ix, map_a, map_b, ws.b_pair_q.as<uint32_t>(), ws.b_pair_d2.as<float>(), ws.p_scale.as<float>(),
        ws.p_sum.as<float>(), ws.b_items.as<uint4>(), nitems, nitems + 1, ws.b_off.as<uint32_t>(),
        ws.p_rowbase.as<unsigned long long>(), ws.p_prox.as<__half>(), ws.p_pscale.as<float>(),
        reinterpret_cast<unsigned long long*>(nitems + 2), ws.err.as<uint32_t>());
    E8QC_CUDA(cudaGetLastError());
    ws.mark_scan(true, s);
}

void launch_scan(const DevIndex& ix, Workspace& ws, size_t a_rows, size_t plane_slots, cudaStream_t s) {
    const CUtensorMap map_a = plane_map(ws.p_a8.p, a_rows / 8, ix.pd, 16);
    const CUtensorMap map_b = plane_map(ix.proxy, plane_slots / 8, ix.pd, 32);
    switch (ws.stages) {
        case 4: launch_scan_stages<4>(ix, ws, map_a, map_b, s); break;
        case 8: launch_scan_stages<8>(ix, ws, map_a, map_b, s); break;
        default: launch_scan_stages<6>(ix, ws, map_a, map_b, s); break;
    }
}

// Per-query selection + exact rescoring of one chunk of queries.
template <int FW>
int launch_select_fw(const DevIndex& ix, Workspace& ws, size_t nq, const uint32_t* k_arr, const uint32_t* np_arr,
                     int k_max, int np_max, cudaStream_t s) {
    constexpr int QPB = 4 / FW;
    precision_select_kernel<FW><<<static_cast<unsigned>((nq + QPB - 1) / QPB), 128, 0, s>>>(
        ix, ws.p_prox.as<__half>(), ws.p_rowbase.as<unsigned long long>(), ws.b_off.as<uint32_t>(),
        ws.b_pos.as<uint32_t>(), ws.b_probes.as<uint32_t>(), ws.b_pd2.as<float>(), static_cast<int>(nq), np_arr,
        np_max, k_arr, k_max, ws.p_cand.as<uint32_t>());
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

// Candidate selection (4 warps per query from kFinalWideRows proxy rows per
// query or below kFinalWideBatch queries, else one) and then the exact
// rescoring.
template <int BITS, bool ME8Q = false>
int launch_final(const DevIndex& ix, const Me8qView& mv, Workspace& ws, const float* rq, size_t nq,
                 const uint32_t* k_arr, const uint32_t* np_arr, int k_max, int np_max, int out_stride,
                 uint32_t* out_ids, float* out_d, size_t rows_per_query, cudaStream_t s) {
    int launches = (rows_per_query >= kFinalWideRows || nq < kFinalWideBatch)
                       ? launch_select_fw<4>(ix, ws, nq, k_arr, np_arr, k_max, np_max, s)
                       : launch_select_fw<1>(ix, ws, nq, k_arr, np_arr, k_max, np_max, s);
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    constexpr int REP = table_rep(BITS);
    // four queries per block when each has one unit of 32 candidates, else one
    // (its up to four units spread over the block's warps)
    const bool one = precision_candidates(k_max) > 32;
    const int qpb = one ? 1 : 4;
    const size_t fsmem = ((ME8Q ? 0 : static_cast<size_t>(2) * (1 << BITS) * REP) +
                          static_cast<size_t>(qpb) * ix.pd + static_cast<size_t>(qpb) * kMaxK * 2) *
                         4;
    static size_t fconfigured[2][64] = {};
    if (fsmem > 48 * 1024 && fconfigured[one][dev & 63] < fsmem) {
        if (one)
            E8QC_CUDA(cudaFuncSetAttribute(precision_rescore_kernel<BITS, ME8Q, 1>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(fsmem)));
        else
            E8QC_CUDA(cudaFuncSetAttribute(precision_rescore_kernel<BITS, ME8Q, 4>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(fsmem)));
        fconfigured[one][dev & 63] = fsmem;
    }
    const unsigned grid = static_cast<unsigned>((nq + qpb - 1) / qpb);
    if (one)
        precision_rescore_kernel<BITS, ME8Q, 1><<<grid, 128, fsmem, s>>>(
            ix, mv, rq, ws.p_cand.as<uint32_t>(), ws.b_probes.as<uint32_t>(), ws.b_pd2.as<float>(),
            static_cast<int>(nq), np_arr, np_max, k_arr, k_max, out_stride, out_ids, out_d);
    else
        precision_rescore_kernel<BITS, ME8Q, 4><<<grid, 128, fsmem, s>>>(
            ix, mv, rq, ws.p_cand.as<uint32_t>(), ws.b_probes.as<uint32_t>(), ws.b_pd2.as<float>(),
            static_cast<int>(nq), np_arr, np_max, k_arr, k_max, out_stride, out_ids, out_d);
    E8QC_CUDA(cudaGetLastError());
    return launches + 1;
}

template <int BITS>
int launch_build_proxy_bits(const DevIndex& ix, int ntiles, const int8_t* lut, uint4* plane, cudaStream_t s) {
    const int nslots = ntiles * 32;
    dim3 g(static_cast<unsigned>((nslots + 255) / 256), static_cast<unsigned>(ix.pd / kPK));
    build_proxy_kernel<BITS><<<g, 256, 0, s>>>(ix, nslots, lut, reinterpret_cast<unsigned char*>(plane));
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

}  // namespace

// The level table as the device holds it (fp32 level / sqrt(Dpad)), its
// int8 step and the quantised table (branch-major).
std::vector<int8_t> proxy_table(int bits, int pd, float* step) {
    const int q = 1 << bits;
    std::vector<float> tab(2 * static_cast<size_t>(q));
    float amax = 0.0f;
    for (int br = 0; br < 2; ++br) {
        const std::vector<double> lev = branch_levels(bits, br);
        for (int d = 0; d < q; ++d) {
            tab[br * q + d] = static_cast<float>(lev[d] / std::sqrt(static_cast<double>(pd)));
            amax = std::max(amax, std::fabs(tab[br * q + d]));
        }
    }
    *step = amax > 0.0f ? amax / 127.0f : 1.0f;
    std::vector<int8_t> lut(tab.size());
    for (size_t e = 0; e < tab.size(); ++e) {
        const long v = std::lrint(static_cast<double>(tab[e]) / static_cast<double>(*step));
        lut[e] = static_cast<int8_t>(std::max(-127L, std::min(127L, v)));
    }
    return lut;
}

float precision_proxy_step(int bits, int pd) {
    float step = 1.0f;
    proxy_table(bits, pd, &step);
    return step;
}

size_t proxy_plane_bytes(const DevIndex& ix, size_t ntiles) {
    return (ntiles * 32 + kPN) * static_cast<size_t>(ix.pd);
}

int launch_build_proxy(const DevIndex& ix, int ntiles, uint4* plane, cudaStream_t s) {
    if (ix.pd % kPK != 0) fail(E8QC_EINVAL, "precision search needs the padded dimension to be a multiple of 64");
    if (ix.bits < 1 || ix.bits > 13) fail(E8QC_EINVAL, "bits out of range");
    // the slots past the last tile are read by the last MMA tile: zero them
    E8QC_CUDA(cudaMemsetAsync(plane, 0, proxy_plane_bytes(ix, ntiles), s));
    float step = 1.0f;
    const std::vector<int8_t> lut_h = proxy_table(ix.bits, ix.pd, &step);
    DevBuf lut;  // one-time build: freed after the kernel below has run
    lut.upload(lut_h.data(), lut_h.size(), s);
    int launches = 0;
    switch (ix.bits) {
#define E8QC_CASE(b) \
    case b: launches = 1 + launch_build_proxy_bits<b>(ix, ntiles, lut.as<int8_t>(), plane, s); break;
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    E8QC_CUDA(cudaStreamSynchronize(s));
    return launches;
}

size_t vcodes_bytes(const DevIndex& ix, size_t ntiles) {
    return ntiles * 32 * static_cast<size_t>(ix.nch) * sizeof(uint4);
}

int launch_vcodes(const DevIndex& ix, int ntiles, uint4* out, cudaStream_t s) {
    const size_t nslots = static_cast<size_t>(ntiles) * 32;
    if (nslots == 0) return 0;
    const size_t total = nslots * ix.nch;
    const unsigned grid = static_cast<unsigned>(std::min<size_t>((total + 255) / 256, 148 * 16));
    vcodes_kernel<<<grid, 256, 0, s>>>(ix.codes, nslots, ix.nch, out);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int precision_candidates(int k) { return candidates_for(k); }

size_t precision_row_scratch(size_t nq, size_t rows_per_query) {
    const size_t per_q = std::max<size_t>(1, rows_per_query) * sizeof(__half);
    const size_t chunk = std::max<size_t>(1, std::min(nq, kScratchBudget / per_q));
    return chunk * (per_q + static_cast<size_t>(kMaxK) * 4);  // proxy rows + candidate slots
}

int precision_search(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                     const uint32_t* np_arr, size_t k, size_t nprobe, size_t out_stride, uint32_t* out_ids,
                     float* out_d, size_t rows_per_query, cudaStream_t s, const Me8qView* me8q) {
    if (nq == 0) return 0;
    if (ix.pd % kPK != 0) fail(E8QC_EINVAL, "precision search needs the padded dimension to be a multiple of 64");
    if (ix.proxy == nullptr) fail(E8QC_ESTATE, "precision search needs the proxy plane (launch_build_proxy)");
    if (me8q == nullptr && ix.vcodes == nullptr)
        fail(E8QC_ESTATE, "precision search needs the slot-major codes (launch_vcodes)");
    // the epilogue forms S' = (coef / qs) * (2 S8 + 0): E8Q coef = step / 2
    // (one table step for every vector); ME8Q coef = 1/2 with the slot's own
    // step in the g1 plane (hsum in h3)
    const float coef = me8q ? 0.5f : 0.5f * ix.proxy_scale;
    const Me8qView none{};
    // proxy rows of a chunk of queries stay within the scratch budget
    const size_t per_q = std::max<size_t>(1, rows_per_query) * sizeof(__half);
    const size_t chunk = std::max<size_t>(1, std::min(nq, kScratchBudget / per_q));
    ws.ensure_err();
    int launches = 0;
    for (size_t off = 0; off < nq; off += chunk) {
        const size_t n = std::min(chunk, nq - off);
        const float* rqc = rq + off * ix.pd;
        const uint32_t* kc = k_arr ? k_arr + off : nullptr;
        const uint32_t* npc = np_arr ? np_arr + off : nullptr;
        ws.mark_prep(false, s);
        launches += batched_prepare(ix, ws, rqc, n, npc, nprobe, 0, kPM, 8, s);
        ws.mark_prep(true, s);
        const size_t pslots = n * nprobe + static_cast<size_t>(7) * ix.nlist;
        const size_t arows = (pslots + 7) / 8 * 8 + kPM;  // an item reads up to 128 rows from its start
        ws.p_q8.ensure(n * static_cast<size_t>(ix.pd));
        ws.p_scale.ensure(n * 4);
        ws.p_sum.ensure(n * 4);
        ws.p_pscale.ensure(n * 4);
        ws.p_rowbase.ensure(static_cast<size_t>(ix.nlist) * 8);
        ws.p_prox.ensure(n * per_q);
        ws.p_cand.ensure(n * static_cast<size_t>(kMaxK) * 4);
        ws.p_a8.ensure(arows * ix.pd);
        rowbase_kernel<<<1, 1024, 0, s>>>(ws.b_cnt.as<uint32_t>(), ix.tile_begin, ix.nlist,
                                          ws.p_rowbase.as<unsigned long long>());
        quantize_kernel<<<static_cast<unsigned>(n), 256, 0, s>>>(
            rqc, ix.pd, coef, 0, ws.p_q8.as<int8_t>(), ws.p_scale.as<float>(), ws.p_sum.as<float>(),
            ws.b_pd2.as<float>(), npc, static_cast<int>(nprobe), static_cast<int>(nprobe), ws.p_pscale.as<float>());
        const size_t ga = arows * (ix.pd / 16);
        gather_a8_kernel<<<static_cast<unsigned>((ga + 255) / 256), 256, 0, s>>>(
            ws.p_q8.as<int8_t>(), ws.b_pair_q.as<uint32_t>(), pslots, arows, ix.pd, ws.p_a8.as<unsigned char>());
        E8QC_CUDA(cudaGetLastError());
        launch_scan(ix, ws, arows, static_cast<size_t>(ix.ntiles) * 32 + kPN, s);
        launches += 4;
        ws.mark_final(false, s);
        if (me8q) {
            launches += launch_final<1, true>(ix, *me8q, ws, rqc, n, kc, npc, static_cast<int>(k),
                                              static_cast<int>(nprobe), static_cast<int>(out_stride),
                                              out_ids + off * out_stride, out_d + off * out_stride, rows_per_query,
                                              s);
            ws.mark_final(true, s);
            continue;
        }
        switch (ix.bits) {
#define E8QC_CASE(b)                                                                                             \
    case b:                                                                                                      \
        launches += launch_final<b>(ix, none, ws, rqc, n, kc, npc, static_cast<int>(k), static_cast<int>(nprobe), \
                                    static_cast<int>(out_stride), out_ids + off * out_stride,                    \
                                    out_d + off * out_stride, rows_per_query, s);                                \
        break;
            E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
            E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
            E8QC_CASE(13)
#undef E8QC_CASE
            default: fail(E8QC_EINVAL, "bits out of range");
        }
        ws.mark_final(true, s);
    }
    return launches;
}

}  // namespace e8qc
