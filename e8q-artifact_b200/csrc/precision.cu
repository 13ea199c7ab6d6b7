// Precision search path: INT8 tensor-core candidate generation + exact
// rescoring.
//
// The lattice code of a vector is a small integer point: coordinate i of a
// block is t_i + eta with t_i the signed digit and eta = 1/4 + br/2, so
// 2*(t + eta) = (2t + br) + 1/2. p = (2t + br) >> max(0, bits - 7) is an exact
// int8 for rates <= 7 and keeps the top 8 bits above. The query is quantised
// to int8 with a per-query scale qs, S8 = sum_i q8_i * p_i runs on tcgen05
// kind::i8 with int32 accumulation in TMEM, and since the level tables are
// close to linear in t + eta near the centre,
//   S ~ S' = alpha * shift / (4 qs) * (2 S8 + sum(q8)),   shift = 2^max(0, bits-7)
// (alpha: a weighted least-squares fit of table against t + eta). The proxy
// distance D' = (d2 + h3) - 2*g1*S' ranks candidates: each query keeps its
// top-C by D' per probed list, and a final kernel merges them per query,
// rescores the C candidates with the exact estimator of the plain scan
// (src/simd/e8q_search_generic.cpp:58-66; same table and per-block FMA chain,
// blocks summed in order into two alternating accumulators) and keeps the
// top-k. A rescored distance depends only on (query, vector), so results do
// not depend on what else is in the batch.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "decode_accum.cuh"
#include "device_common.cuh"
#include "internal.h"
#include "precision.h"
#include "scan_plain.h"
#include "tc.cuh"
#include "tma.cuh"
#include "workspace.h"

namespace e8qc {

namespace {

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

constexpr int kPT = 128;  // threads (one warpgroup: 4 warps x 32 TMEM lanes)
constexpr int kPM = 128;  // queries per MMA tile (M)
constexpr int kPN = 256;  // vectors per MMA tile (N)
constexpr int kPK = 64;   // dimensions per staged K-chunk (2 MMAs of K = 32)
constexpr uint32_t kCols = 256;  // TMEM columns: one int32 accumulator per vector

// Per-query int8 quantisation: q8 = rint(q * 127 / max|q|); per-query factor
// coef / qs and sum(q8).
__global__ void quantize_kernel(const float* __restrict__ rq, int pd, float coef, int8_t* __restrict__ q8,
                                float* __restrict__ qscale, float* __restrict__ qsum) {
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
        qsum[blockIdx.x] = static_cast<float>(s);
    }
}

// 32-bit word `w` of the code stream of the vector in lane `lane` of tile gt.
__device__ __forceinline__ uint32_t code_word(const DevIndex& ix, uint32_t gt, int lane, int w) {
    const uint32_t* base =
        reinterpret_cast<const uint32_t*>(ix.codes + (static_cast<size_t>(gt) * ix.nch + (w >> 2)) * 32 + lane);
    return __ldg(base + (w & 3));
}

// Proxy integers of one block (8 dims) as 8 packed int8.
template <int BITS>
__device__ __forceinline__ uint2 block_proxy(const uint32_t* w, int base) {
    constexpr int SH = BITS > 7 ? BITS - 7 : 0;
    uint32_t dg[8];
    const int br = decode_block<BITS>(w, base, dg);
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int t = static_cast<int>(dg[i]) - ((dg[i] >> (BITS - 1)) ? (1 << BITS) : 0);
        const uint32_t p = static_cast<uint32_t>((2 * t + br) >> SH) & 0xFFu;  // arithmetic shift: floor
        if (i < 4) lo |= p << (8 * i);
        else hi |= p << (8 * (i - 4));
    }
    return make_uint2(lo, hi);
}

// Persistent proxy scan over work items (one list, up to 128 queries): for
// each 256-vector tile of the list, K-chunks of 64 dimensions are staged in
// shared memory (queries: int8 copies; vectors: decoded proxy integers) in the
// K-major no-swizzle layout, double-buffered, and one thread issues the two
// kind::i8 MMAs of a chunk into the 128 x 256 int32 accumulator in TMEM. The
// epilogue reads the accumulator row of its query (thread r = TMEM lane r)
// and keeps the query's top-C proxy distances in shared memory.
template <int BITS>
__global__ void __launch_bounds__(kPT, 1) precision_scan_kernel(
    DevIndex ix, const int8_t* __restrict__ q8, const float* __restrict__ qscale, const float* __restrict__ qsum,
    const uint4* __restrict__ items, const uint32_t* __restrict__ n_items, uint32_t* __restrict__ head,
    const uint32_t* __restrict__ pair_q, const float* __restrict__ pair_d2, int C, float* __restrict__ part_d,
    uint32_t* __restrict__ part_slot, unsigned long long* __restrict__ cand_count, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char psm[];
    unsigned char* sA = psm;                                      // 2 x kPM x kPK
    unsigned char* sB = psm + 2 * kPM * kPK;                      // 2 x kPN x kPK
    float* tc_d = reinterpret_cast<float*>(sB + 2 * kPN * kPK);  // kPM x C
    uint32_t* tc_i = reinterpret_cast<uint32_t*>(tc_d + kPM * C);
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint4 s_item;
    __shared__ uint32_t s_q[kPM];
    __shared__ float s_d2[kPM], s_sc[kPM], s_sum[kPM];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int pd = ix.pd, nK = pd / kPK;
    if (warp == 0) {
        tc::tmem_alloc(&s_tmem, kCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        fence_barrier_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = tc::idesc_i8(kPM, kPN);
    const uint32_t sbo = (kPK / 16) * 128u;
    const uint32_t NI = *n_items;
    uint32_t ck = 0;  // K-chunks committed so far: buffer ck & 1, phase (ck >> 1) & 1
    bool ok = true;   // uniform across the CTA (every decision goes through a barrier)
    for (;;) {
        __syncthreads();
        if (tid == 0) {
            const uint32_t it = atomicAdd(head, 1u);
            s_item = it < NI ? items[it] : make_uint4(0xFFFFFFFFu, 0, 0, 0);
        }
        __syncthreads();
        const uint4 item = s_item;
        if (item.x == 0xFFFFFFFFu) break;
        const uint32_t L = item.x, pbase = item.y;
        const int m = static_cast<int>(item.z);
        {
            const bool in = tid < m;
            const uint32_t qq = in ? pair_q[pbase + tid] : 0u;
            s_q[tid] = qq;
            s_d2[tid] = in ? pair_d2[pbase + tid] : 0.0f;
            s_sc[tid] = in ? qscale[qq] : 0.0f;
            s_sum[tid] = in ? qsum[qq] : 0.0f;
        }
        for (int e = tid; e < kPM * C; e += kPT) {
            tc_d[e] = inf_f();
            tc_i[e] = 0xFFFFFFFFu;
        }
        const uint32_t len = ix.list_len[L];
        const uint32_t tile0 = ix.tile_begin[L];
        if (tid == 0) {
            atomicAdd(cand_count, static_cast<unsigned long long>(len) * m);  // (query, vector) pairs
            atomicAdd(cand_count + 1, static_cast<unsigned long long>(len));  // vectors read
        }
        __syncthreads();
        float thr = inf_f();  // this thread's query: C-th best proxy distance so far
        const int r = tid;    // query row == TMEM lane
        for (uint32_t v0 = 0; v0 < len && ok; v0 += kPN) {
            for (int kc = 0; kc < nK; ++kc, ++ck) {
                const int b = static_cast<int>(ck & 1u);
                bool mine = true;
                if (ck >= 2) mine = mbar_wait_bounded(&s_bar[b], ((ck - 2) >> 1) & 1u);  // buffer b free
                unsigned char* A = sA + b * kPM * kPK;
                unsigned char* Bm = sB + b * kPN * kPK;
                // A: 128 query rows x 64 int8
                for (int e = tid; e < kPM * 4; e += kPT) {
                    const int row = e >> 2, c16 = e & 3;
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (row < m)
                        v = *reinterpret_cast<const uint4*>(q8 + static_cast<size_t>(s_q[row]) * pd + kc * kPK +
                                                            c16 * 16);
                    *reinterpret_cast<uint4*>(A + tc::il_offset(row, c16 * 16, kPK)) = v;
                }
                // B: 256 vectors x 8 blocks of proxy integers
                for (int e = tid; e < kPN * 8; e += kPT) {
                    const int vv = e >> 3, blk = e & 7;
                    const uint32_t vi = v0 + vv;
                    uint2 pv = make_uint2(0, 0);
                    if (vi < len) {
                        const uint32_t gt = tile0 + (vi >> 5);
                        const int vl = static_cast<int>(vi & 31u);
                        const int bit0 = (kc * 8 + blk) * 8 * BITS;
                        uint32_t w[6];
#pragma unroll
                        for (int j = 0; j < 5; ++j)
                            w[j] = (j * 32 < (bit0 & 31) + 8 * BITS) ? code_word(ix, gt, vl, (bit0 >> 5) + j) : 0u;
                        w[5] = 0u;
                        pv = block_proxy<BITS>(w, bit0 & 31);
                    }
                    *reinterpret_cast<uint2*>(Bm + tc::il_offset(vv, blk * 8, kPK)) = pv;
                }
                tc::fence_smem_to_async();
                tc::fence_before_sync();
                ok = __syncthreads_and(mine ? 1 : 0) != 0;
                tc::fence_after_sync();
                if (!ok) break;
                if (tid == 0) {
                    const uint32_t a0 = tc::saddr(A), b0 = tc::saddr(Bm);
#pragma unroll
                    for (int s = 0; s < kPK / 32; ++s)
                        tc::mma_i8(tmem, tc::smem_desc(a0 + 256u * s, 128u, sbo),
                                   tc::smem_desc(b0 + 256u * s, 128u, sbo), idesc, (kc > 0 || s > 0) ? 1u : 0u);
                    tc::mma_commit(&s_bar[b]);
                }
            }
            if (!ok) break;
            // the tile's last commit covers all its MMAs
            const uint32_t last = ck - 1;
            const bool done = mbar_wait_bounded(&s_bar[last & 1u], (last >> 1) & 1u);
            ok = __syncthreads_and(done ? 1 : 0) != 0;
            if (!ok) break;
            tc::fence_after_sync();
            const float sc = s_sc[r], sum = s_sum[r], d2 = s_d2[r];
            float* ld = tc_d + r * C;
            uint32_t* li = tc_i + r * C;
            for (int c0 = 0; c0 < kPN; c0 += 8) {
                uint32_t acc[8];
                tc::tmem_ld8(tmem + ((static_cast<uint32_t>(warp) * 32u) << 16) + static_cast<uint32_t>(c0), acc);
                tc::tmem_ld_wait();
                if (r < m) {
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const uint32_t vi = v0 + c0 + j;
                        if (vi >= len) break;
                        const uint32_t slot = (tile0 + (vi >> 5)) * 32u + (vi & 31u);
                        const float g1 = __ldg(ix.g1 + slot), h3 = __ldg(ix.h3 + slot);
                        const float Sp = sc * __fmaf_rn(2.0f, static_cast<float>(static_cast<int>(acc[j])), sum);
                        const float dp = __fmaf_rn(-__fmul_rn(2.0f, g1), Sp, __fadd_rn(d2, h3));
                        if (dp < thr) {  // sorted insertion into this query's list
                            int pos = C - 1;
                            while (pos > 0 && ld[pos - 1] > dp) {
                                ld[pos] = ld[pos - 1];
                                li[pos] = li[pos - 1];
                                --pos;
                            }
                            ld[pos] = dp;
                            li[pos] = slot;
                            thr = ld[C - 1];
                        }
                    }
                }
            }
            tc::fence_before_sync();
            __syncthreads();  // TMEM reads done before the next tile's MMAs overwrite it
        }
        if (!ok) break;
        // the item's per-pair candidate lists
        for (int e = tid; e < m * C; e += kPT) {
            const int q = e / C, j = e - q * C;
            const size_t o = static_cast<size_t>(pbase + q) * C + j;
            part_d[o] = tc_d[q * C + j];
            part_slot[o] = tc_i[q * C + j];
        }
    }
    if (!ok) {
        // a wait gave up: report, give in-flight MMAs one more bounded wait
        if (tid == 0) atomicOr(err, kErrWaitTimeout);
        if (ck > 0) (void)mbar_wait_bounded(&s_bar[(ck - 1) & 1u], ((ck - 1) >> 1) & 1u, 256u);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kCols);
}

// Per query (one warp): merge the query's per-list candidate lists into its
// top-C by proxy distance, rescore those exactly, keep the top-k.
template <int BITS>
__global__ void __launch_bounds__(128) precision_final_kernel(
    DevIndex ix, const float* __restrict__ rq, const float* __restrict__ part_d,
    const uint32_t* __restrict__ part_slot, int C, const uint32_t* __restrict__ pos_of,
    const uint32_t* __restrict__ probes, const float* __restrict__ pd2, int nq, const uint32_t* __restrict__ np_arr,
    int np_max, const uint32_t* __restrict__ k_arr, int k_uniform, int out_stride, uint32_t* __restrict__ out_ids,
    float* __restrict__ out_d) {
    constexpr int Q = 1 << BITS;
    constexpr int REP = table_rep(BITS);
    constexpr int GBL = group_blocks(BITS), GCH = group_chunks(BITS);
    constexpr int TCH = (64 * BITS + 127) / 128;
    extern __shared__ __align__(16) float fsm[];
    float* tabrep = fsm;               // 2*Q*REP
    float* sq = tabrep + 2 * Q * REP;  // 4 warps x pd
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < 2 * Q * REP; e += blockDim.x) tabrep[e] = ix.tab[e / REP];
    const int q = blockIdx.x * 4 + warp;
    const int pd = ix.pd;
    float* myq = sq + warp * pd;
    if (q < nq)
        for (int i = lane; i < pd; i += 32) myq[i] = rq[static_cast<size_t>(q) * pd + i];
    __syncthreads();
    if (q >= nq) return;
    const int np = np_arr ? static_cast<int>(np_arr[q]) : np_max;
    const int kq = k_arr ? static_cast<int>(k_arr[q]) : k_uniform;
    // 1. top-C candidates of this query by proxy distance (slot as tie-break)
    WarpTopK cand;
    cand.init(C);
    for (int p = 0; p < np; ++p) {
        const size_t base = static_cast<size_t>(pos_of[static_cast<size_t>(q) * np_max + p]) * C;
        for (int j0 = 0; j0 < C; j0 += 32) {
            const int j = j0 + lane;
            const bool in = j < C;
            const float dd = in ? part_d[base + j] : inf_f();
            const uint32_t ss = in ? part_slot[base + j] : 0xFFFFFFFFu;
            cand.offer_pair(dd, ss, in && ss != 0xFFFFFFFFu);
        }
    }
    // 2. exact rescoring of candidate (s, lane); 3. top-k by exact distance
    WarpTopK top;
    top.init(kq);
    const uint32_t tb_addr = static_cast<uint32_t>(__cvta_generic_to_shared(tabrep)) + (lane % REP) * 4u;
    const float4* sq4 = reinterpret_cast<const float4*>(myq);
    const uint32_t* pr = probes + static_cast<size_t>(q) * np_max;
    const int ng = (pd / 8) / GBL;
    const bool tail = ((pd / 8) % GBL) != 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        if (s * 32 >= C) break;
        const uint32_t slot = cand.id[s];
        const bool live = s * 32 + lane < C && slot != 0xFFFFFFFFu;
        float dist = inf_f();
        uint32_t gid = 0xFFFFFFFFu;
        if (live) {
            const uint32_t tile = slot >> 5;
            const int vl = static_cast<int>(slot & 31u);
            const uint4* tp = ix.codes + static_cast<size_t>(tile) * ix.nch * 32;
            float acc0 = 0.0f, acc1 = 0.0f;
            for (int g = 0; g < ng; ++g)
                accumulate_blocks<BITS, GBL, GCH>(tp + g * GCH * 32, vl, sq4, g * GBL, tb_addr, acc0, acc1);
            if (tail) accumulate_blocks<BITS, 8, TCH>(tp + ng * GCH * 32, vl, sq4, ng * GBL, tb_addr, acc0, acc1);
            const float S = __fadd_rn(acc0, acc1);
            // d2 of (query, the candidate's list): the query's probes are in list order
            const uint32_t list = ix.list_of_tile[tile];
            int lo = 0, hi = np;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (pr[mid] <= list) lo = mid;
                else hi = mid;
            }
            const float d2 = pd2[static_cast<size_t>(q) * np_max + lo];
            dist = __fmaf_rn(-__fmul_rn(2.0f, __ldg(ix.g1 + slot)), S, __fadd_rn(d2, __ldg(ix.h3 + slot)));
            gid = __ldg(ix.ids + slot);
        }
        top.offer_pair(dist, gid, live);
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int j = s * 32 + lane;
        if (j < out_stride) {
            const bool in = j < kq;
            out_d[static_cast<size_t>(q) * out_stride + j] = in ? top.d[s] : inf_f();
            out_ids[static_cast<size_t>(q) * out_stride + j] = in ? top.id[s] : 0xFFFFFFFFu;
        }
    }
}

size_t scan_smem(int C) { return static_cast<size_t>(2) * kPM * kPK + 2 * kPN * kPK + static_cast<size_t>(kPM) * C * 8; }

template <int BITS>
int launch_precision(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                     const uint32_t* np_arr, int k_max, int np_max, int C, int out_stride, uint32_t* out_ids,
                     float* out_d, cudaStream_t s) {
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    const size_t smem = scan_smem(C);
    static size_t configured[64] = {};
    if (configured[dev & 63] < smem) {
        E8QC_CUDA(cudaFuncSetAttribute(precision_scan_kernel<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        configured[dev & 63] = smem;
    }
    int sms = 148, per_sm = 1;
    E8QC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    E8QC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, precision_scan_kernel<BITS>, kPT, smem));
    per_sm = std::max(1, std::min(per_sm, 2));  // 2 x 256 TMEM columns fill an SM
    uint32_t* nitems = ws.b_nitems.as<uint32_t>();
    ws.mark_scan(false, s);
    precision_scan_kernel<BITS><<<sms * per_sm, kPT, smem, s>>>(
        ix, ws.p_q8.as<int8_t>(), ws.p_scale.as<float>(), ws.p_sum.as<float>(), ws.b_items.as<uint4>(), nitems,
        nitems + 1, ws.b_pair_q.as<uint32_t>(), ws.b_pair_d2.as<float>(), C, ws.b_part_d.as<float>(),
        ws.b_part_id.as<uint32_t>(), reinterpret_cast<unsigned long long*>(nitems + 2), ws.err.as<uint32_t>());
    E8QC_CUDA(cudaGetLastError());
    ws.mark_scan(true, s);
    constexpr int REP = table_rep(BITS);
    const size_t fsmem = (static_cast<size_t>(2) * (1 << BITS) * REP + 4 * static_cast<size_t>(ix.pd)) * 4;
    static size_t fconfigured[64] = {};
    if (fsmem > 48 * 1024 && fconfigured[dev & 63] < fsmem) {
        E8QC_CUDA(cudaFuncSetAttribute(precision_final_kernel<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(fsmem)));
        fconfigured[dev & 63] = fsmem;
    }
    precision_final_kernel<BITS><<<static_cast<unsigned>((nq + 3) / 4), 128, fsmem, s>>>(
        ix, rq, ws.b_part_d.as<float>(), ws.b_part_id.as<uint32_t>(), C, ws.b_pos.as<uint32_t>(),
        ws.b_probes.as<uint32_t>(), ws.b_pd2.as<float>(), static_cast<int>(nq), np_arr, np_max, k_arr, k_max,
        out_stride, out_ids, out_d);
    E8QC_CUDA(cudaGetLastError());
    return 2;
}

}  // namespace

double precision_alpha(int bits, int pd) {
    const int q = 1 << bits;
    const double s = fixed_scale(bits);
    double sxy = 0.0, sxx = 0.0;
    for (int br = 0; br < 2; ++br) {
        const std::vector<double> lev = branch_levels(bits, br);
        for (int d = 0; d < q; ++d) {
            const int t = d >= q / 2 ? d - q : d;
            const double x = t + 0.25 + 0.5 * br;
            const double y = lev[d] / std::sqrt(static_cast<double>(pd));
            const double w = std::exp(-lev[d] * lev[d] / (2.0 * s * s));
            sxy += w * x * y;
            sxx += w * x * x;
        }
    }
    return sxx > 0.0 ? sxy / sxx : 0.0;
}

int precision_candidates(int k) { return std::min(kMaxK, std::max(64, 4 * k)); }

int precision_search(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                     const uint32_t* np_arr, size_t k, size_t nprobe, size_t out_stride, uint32_t* out_ids,
                     float* out_d, cudaStream_t s) {
    if (nq == 0) return 0;
    if (ix.pd % kPK != 0) fail(E8QC_EINVAL, "precision search needs the padded dimension to be a multiple of 64");
    const int C = precision_candidates(static_cast<int>(k));
    int launches = batched_prepare(ix, ws, rq, nq, np_arr, nprobe, static_cast<size_t>(C), kPM, s);
    ws.p_q8.ensure(nq * static_cast<size_t>(ix.pd));
    ws.p_scale.ensure(nq * 4);
    ws.p_sum.ensure(nq * 4);
    ws.ensure_err();
    const int shift = ix.bits > 7 ? (1 << (ix.bits - 7)) : 1;
    const float coef = static_cast<float>(precision_alpha(ix.bits, ix.pd) * shift / 4.0);
    quantize_kernel<<<static_cast<unsigned>(nq), 256, 0, s>>>(rq, ix.pd, coef, ws.p_q8.as<int8_t>(),
                                                              ws.p_scale.as<float>(), ws.p_sum.as<float>());
    E8QC_CUDA(cudaGetLastError());
    ++launches;
    switch (ix.bits) {
#define E8QC_CASE(b)                                                                                                 \
    case b:                                                                                                          \
        launches += launch_precision<b>(ix, ws, rq, nq, k_arr, np_arr, static_cast<int>(k), static_cast<int>(nprobe), \
                                        C, static_cast<int>(out_stride), out_ids, out_d, s);                         \
        break;
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    return launches;
}

}  // namespace e8qc
