// Batch routing on the int8 tensor cores, with the exact keys of the fp64
// route (src/index/ivf_route.cpp:9-27, src/simd/kernels_generic.cpp:13-33:
// dot accumulated in fp64, d2 = qn2 + cn2 - 2 * float(dot) clamped at 0,
// key = (bits(d2) << 32) | list id, the nprobe smallest keys).
//
// 1. Slicing (route_slice_kernel): each row x (a rotated query or centroid)
//    is scaled by 127 / 2^e, 2^e > max|x|, and split exactly in fp64 into
//    three int8 slices, X = Q0 + Q1/128 + Q2/128^2 + rho with |Q0| <= 127,
//    |Q1|, |Q2| <= 64 and |rho_i| <= 2^-15, plus the row's norms |Q1|, |Q2|,
//    |Q0 + Q1/128 + Q2/128^2| (rounded up).
// 2. Bound GEMM (route_tc_kernel): tcgen05 kind::i8 products of the slices
//    with exact int32 accumulation, the six with t + u <= 2 summed by weight
//    into three TMEM accumulators (P00, P01 + P10, P02 + P11 + P20). The
//    epilogue forms the approximate dot in fp64 and a rigorous bound on its
//    error (dropped slice products by Cauchy-Schwarz on the slice norms, the
//    residuals rho, the rounding of the reference's own fp64 dot and of the
//    float key arithmetic, all with slack), and writes per (query, list) a
//    float interval [lo, hi] that holds the list's exact d2.
// 3. Selection: U = the nprobe-th smallest hi, and every list with lo <= U
//    is a candidate (route_cand_kernel; a list with lo > U has at least nprobe
//    lists with smaller keys); each candidate's exact key is computed with the
//    same sequential fp64 FMA chain over the dimensions as route_gemm_kernel
//    (route_rekey_kernel), and the nprobe smallest keys are taken
//    (route_pick_kernel). The result -- probes in list
//    order, their d2 and the per-list pair counts -- is that of the fp64 route
//    GEMM, bit for bit.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "device_common.cuh"
#include "internal.h"
#include "precision.h"
#include "route_tc.h"
#include "tc.cuh"
#include "tma.cuh"
#include "workspace.h"

namespace e8qc {

namespace {

constexpr int kRT = 128;                             // rows per tile on both sides (queries: TMEM lanes)
constexpr int kRK = 64;                              // K bytes per chunk
constexpr int kRSlab = kRT * kRK;                    // 8 KB: one slice of one side for one chunk
constexpr int kRStageBytes = 6 * kRSlab;             // 3 query + 3 list slices
constexpr int kRStages = 4;
constexpr int kRThreads = 192;
constexpr uint32_t kRCols = 512;                     // 3 accumulators x 128 columns, rounded to a power of two
constexpr int kRouteTcMaxLists = 4096;
constexpr int kRouteTcMaxDim = 4096;
constexpr int kSelThreads = 128;  // threads of the per-query candidate and pick kernels
constexpr int kRkThreads = 128;   // exact-key kernel: 4 warps per CTA, one unit per warp at a time
constexpr int kRkStages = 4;      // 32-dimension blocks per warp ring (3 in flight)
constexpr int kRkBlocksPerSm = 3; // 3 x 4 x 16.9 KB of rings per SM

// One warp per row of a plane of rows_pad rows (slice t at rows t*rows_pad..):
// rows < n hold src's row, the rest are zero. meta[r] = (2^e, |Q1|, |Q2|, |Xhat|).
__global__ void route_slice_kernel(const float* __restrict__ src, int n, int rows_pad, int pd,
                                   int8_t* __restrict__ plane, float4* __restrict__ meta) {
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (r >= rows_pad) return;
    const bool live = r < n;
    const float* row = src + static_cast<size_t>(live ? r : 0) * pd;
    float mx = 0.0f;
    if (live)
        for (int i = lane; i < pd; i += 32) mx = fmaxf(mx, fabsf(row[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
    int e = 0;
    if (mx > 0.0f) (void)frexpf(mx, &e);  // mx < 2^e
    const double f = ldexp(127.0, -e);   // x = row * f is exact (24-bit x 7-bit significands)
    double n1 = 0.0, n2 = 0.0, nx = 0.0;
    bool bad = false;  // a NaN or infinite element: the row gets an unbounded interval
    const size_t slice = static_cast<size_t>(rows_pad) * pd;
    for (int p = lane; p < pd / 16; p += 32) {
        uint32_t w[3][4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            w[0][b] = w[1][b] = w[2][b] = 0u;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int i = p * 16 + b * 4 + k;
                double x = live ? static_cast<double>(row[i]) * f : 0.0;
                if (!(fabs(x) <= 127.0)) {
                    bad = true;
                    x = 0.0;
                }
                const double q0 = rint(x);
                double rr = (x - q0) * 128.0;
                const double q1 = rint(rr);
                rr = (rr - q1) * 128.0;
                const double q2 = rint(rr);
                const double xh = q0 + q1 * 0x1p-7 + q2 * 0x1p-14;
                n1 = __fma_rn(q1, q1, n1);
                n2 = __fma_rn(q2, q2, n2);
                nx = __fma_rn(xh, xh, nx);
                w[0][b] |= static_cast<uint32_t>(static_cast<uint8_t>(static_cast<int8_t>(q0))) << (8 * k);
                w[1][b] |= static_cast<uint32_t>(static_cast<uint8_t>(static_cast<int8_t>(q1))) << (8 * k);
                w[2][b] |= static_cast<uint32_t>(static_cast<uint8_t>(static_cast<int8_t>(q2))) << (8 * k);
            }
        }
        const size_t off = tc::il_offset(r, p * 16, pd);
#pragma unroll
        for (int t = 0; t < 3; ++t)
            *reinterpret_cast<uint4*>(plane + t * slice + off) = make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
    }
    bad = __any_sync(kFull, bad);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n1 += __shfl_xor_sync(kFull, n1, o);
        n2 += __shfl_xor_sync(kFull, n2, o);
        nx += __shfl_xor_sync(kFull, nx, o);
    }
    if (lane == 0) {
        // sums of squares of small integers (and of xh, 38-bit fixed point) carry
        // at most a few ulps of rounding: 2^-40 of slack, then round up
        const double up = 1.0 + 0x1p-40;
        const float inf = __int_as_float(0x7f800000);
        meta[r] = bad ? make_float4(1.0f, inf, inf, inf)
                      : make_float4(ldexpf(1.0f, e), __double2float_ru(__dsqrt_ru(n1 * up)),
                                    __double2float_ru(__dsqrt_ru(n2 * up)), __double2float_ru(__dsqrt_ru(nx * up)));
    }
}

// One 128-query x 128-list tile per CTA. Warp 0 loads the six slices of each
// 64-byte K-chunk by TMA into a kRStages ring, one thread of warp 1 issues the
// six kind::i8 MMAs per 32 bytes of K, warps 2-5 read the three accumulators
// (thread = query row) and write each (query, list) interval. Waits are
// bounded; a timeout sets the error word.
__global__ void __launch_bounds__(kRThreads, 1) route_tc_kernel(
    const __grid_constant__ CUtensorMap map_q, const __grid_constant__ CUtensorMap map_c, int nq, int nlist, int pd,
    int qrows_pad, int crows_pad, const float4* __restrict__ qmeta, const float4* __restrict__ cmeta,
    const float* __restrict__ qn2, const float* __restrict__ cn2, float2* __restrict__ out, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char rsm[];
    __shared__ __align__(8) uint64_t full[kRStages], empty[kRStages], tfull, fin;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ double s_cs[kRT];   // the list's 2^e / 127^2
    __shared__ double s_cr[kRT];   // sqrt(cn2), rounded up
    __shared__ float4 s_cm[kRT];   // (unused, |C1|, |C2|, |Yhat|)
    __shared__ float s_cn2[kRT];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nK = pd / kRK;
    const int q0 = blockIdx.y * kRT, c0 = blockIdx.x * kRT;
    if (warp == 0) {
        tc::tmem_alloc(&s_tmem, kRCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        for (int i = 0; i < kRStages; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(&tfull, 1);
        mbar_init(&fin, 1);
        s_abort = 0;
        fence_barrier_init();
    }
    for (int j = tid; j < kRT; j += blockDim.x) {
        const int c = c0 + j;
        s_cm[j] = c < nlist ? cmeta[c] : make_float4(1.0f, 0.0f, 0.0f, 0.0f);
        s_cn2[j] = c < nlist ? cn2[c] : 0.0f;
        s_cs[j] = static_cast<double>(s_cm[j].x) / 16129.0;
        s_cr[j] = __dsqrt_ru(fmax(static_cast<double>(s_cn2[j]), 0.0));
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = s_tmem;

    if (warp == 0) {
        // ---- producer ----
        int kc = 0;
        for (; kc < nK && !s_abort; ++kc) {
            const int st = kc % kRStages;
            if (kc >= kRStages && !mbar_wait_or_abort(&empty[st], ((kc / kRStages) - 1) & 1u, &s_abort)) break;
            if (lane == 0) {
                unsigned char* base = rsm + st * kRStageBytes;
                mbar_arrive_expect_tx(&full[st], kRStageBytes);
                // 16 row groups x 512 bytes (128 u32 at x = kc * 128) per slice
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    tma_load_2d(base + t * kRSlab, &map_q, kc * 128, (t * qrows_pad + q0) >> 3, &full[st]);
                    tma_load_2d(base + (3 + t) * kRSlab, &map_c, kc * 128, (t * crows_pad + c0) >> 3, &full[st]);
                }
            }
            __syncwarp();
        }
        // copies still in flight land before the CTA can exit
        if (s_abort && lane == 0)
            for (int g = kc > kRStages ? kc - kRStages : 0; g < kc; ++g)
                (void)mbar_wait_bounded(&full[g % kRStages], (g / kRStages) & 1u, 100u);
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_i8(kRT, kRT);
            const uint32_t sbo = (kRK / 16) * 128u;
            bool issued = false;
            for (int kc = 0; kc < nK && !s_abort; ++kc) {
                const int st = kc % kRStages;
                if (!mbar_wait_or_abort(&full[st], (kc / kRStages) & 1u, &s_abort)) break;
                tc::fence_after_sync();
                const uint32_t a0 = tc::saddr(rsm + st * kRStageBytes);
#pragma unroll
                for (int s2 = 0; s2 < kRK / 32; ++s2) {
                    const uint32_t acc = (kc > 0 || s2 > 0) ? 1u : 0u;
                    auto A = [&](int t) { return tc::smem_desc(a0 + t * kRSlab + 256u * s2, 128u, sbo); };
                    auto B = [&](int u) { return tc::smem_desc(a0 + (3 + u) * kRSlab + 256u * s2, 128u, sbo); };
                    tc::mma_i8(tmem, A(0), B(0), idesc, acc);
                    tc::mma_i8(tmem + 128u, A(0), B(1), idesc, acc);
                    tc::mma_i8(tmem + 128u, A(1), B(0), idesc, 1u);
                    tc::mma_i8(tmem + 256u, A(0), B(2), idesc, acc);
                    tc::mma_i8(tmem + 256u, A(1), B(1), idesc, 1u);
                    tc::mma_i8(tmem + 256u, A(2), B(0), idesc, 1u);
                }
                tc::mma_commit(&empty[st]);
                issued = true;
            }
            if (!s_abort) tc::mma_commit(&tfull);
            // every MMA issued has completed before TMEM is released
            if (issued) {
                tc::mma_commit(&fin);
                (void)mbar_wait_bounded(&fin, 0u, 200u);
            }
        }
        __syncwarp();
    } else {
        // ---- epilogue: thread = query row q0 + r ----
        const int q4 = warp & 3;
        const int r = q4 * 32 + lane;
        const int q = q0 + r;
        const float4 qm = q < nq ? qmeta[q] : make_float4(1.0f, 0.0f, 0.0f, 0.0f);
        const double qq = q < nq ? static_cast<double>(qn2[q]) : 0.0;
        const double qr = __dsqrt_ru(fmax(qq, 0.0));
        const double n = static_cast<double>(pd), rn = sqrt(n);
        if (mbar_wait_or_abort(&tfull, 0u, &s_abort)) {
            tc::fence_after_sync();
            for (int cb = 0; cb < kRT; cb += 32) {
                uint32_t acc[3][32];
#pragma unroll
                for (int t = 0; t < 3; ++t)
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj) {
                        uint32_t(&part)[8] = *reinterpret_cast<uint32_t(*)[8]>(acc[t] + 8 * jj);
                        tc::tmem_ld8(tmem + ((static_cast<uint32_t>(q4) * 32u) << 16) + t * 128u + cb + 8 * jj, part);
                    }
                tc::tmem_ld_wait();
                if (q >= nq) continue;
                float2* orow = out + static_cast<size_t>(q) * nlist + c0 + cb;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    if (c0 + cb + j >= nlist) continue;
                    const float4 cm = s_cm[cb + j];
                    const double cc = static_cast<double>(s_cn2[cb + j]);
                    // exact: |P| < 2^25, weights are powers of two, 39 significant bits at most
                    const double S = static_cast<double>(static_cast<int>(acc[0][j])) +
                                     static_cast<double>(static_cast<int>(acc[1][j])) * 0x1p-7 +
                                     static_cast<double>(static_cast<int>(acc[2][j])) * 0x1p-14;
                    const double sc = static_cast<double>(qm.x) * s_cs[cb + j];
                    const double dot = S * sc;
                    // |sum x y - S| over the scaled rows: dropped slice products + residuals
                    const double E = 0x1p-21 * (static_cast<double>(qm.y) * cm.z + static_cast<double>(qm.z) * cm.y) +
                                     0x1p-28 * static_cast<double>(qm.z) * cm.z +
                                     0x1p-15 * rn * (static_cast<double>(qm.w) + cm.w) + n * 0x1p-30;
                    const double err = E * sc * (1.0 + 0x1p-40) + fabs(dot) * 0x1p-48;
                    const double a = qq + cc - 2.0 * dot;
                    // the reference key's own roundings: fp64 dot (n ulps of |q||c|),
                    // float(dot), qn2 + cn2 in float, the fused -2 * dot + (qn2 + cn2)
                    const double e = 2.0 * err + 0x1p-21 * (qq + cc + 2.0 * (fabs(dot) + err) + fabs(a)) +
                                     n * 0x1p-50 * qr * s_cr[cb + j] + 1e-30;
                    // non-finite inputs (a NaN or infinite bound): the list is always a candidate
                    orow[j] = (e <= 1e300 && a == a)
                                  ? make_float2(__double2float_rd(fmax(a - e, 0.0)), __double2float_ru(fmax(a + e, 0.0)))
                                  : make_float2(0.0f, __int_as_float(0x7f800000));
                }
            }
        }
    }
    __syncthreads();
    if (s_abort && tid == 0) atomicOr(err, kErrWaitTimeout);
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, kRCols);
}

// The want-th smallest of n distinct-or-equal keys in shared memory (MSB radix
// select, 8 bits per pass); every thread of the block gets it.
template <typename K>
__device__ K block_select(const K* keys, int n, int want, int* hist, K* s_prefix, int* s_want) {
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
        *s_prefix = 0;
        *s_want = want;
    }
    K mask = 0;
    __syncthreads();
    for (int shift = static_cast<int>(sizeof(K)) * 8 - 8; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += nt) hist[i] = 0;
        __syncthreads();
        const K prefix = *s_prefix;
        for (int c = tid; c < n; c += nt) {
            const K key = keys[c];
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1);
        }
        __syncthreads();
        if (tid < 32) {
            int cnt[8], tot = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                cnt[j] = hist[tid * 8 + j];
                tot += cnt[j];
            }
            int incl = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, incl, o);
                if (tid >= o) incl += y;
            }
            const int excl = incl - tot;
            const int wnt = *s_want;
            const unsigned hit = __ballot_sync(kFull, excl < wnt && incl >= wnt);
            const int owner = __ffs(hit) - 1;
            if (tid == owner) {
                int cum = excl, sel = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (cum + cnt[j] >= wnt) {
                        sel = j;
                        break;
                    }
                    cum += cnt[j];
                }
                *s_prefix = prefix | (static_cast<K>(tid * 8 + sel) << shift);
                *s_want = wnt - cum;
            }
        }
        mask |= static_cast<K>(0xFF) << shift;
        __syncthreads();
    }
    return *s_prefix;
}

// Block-wide exclusive scan of one flag per thread; *total gets the sum.
__device__ int block_scan_flag(int flag, int* sm32, int* total) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    int x = flag;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm32[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int v = lane < nw ? sm32[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, v, o);
            if (lane >= o) v += y;
        }
        sm32[lane] = v;
    }
    __syncthreads();
    const int before = (warp > 0 ? sm32[warp - 1] : 0) + x - flag;
    *total = sm32[nw - 1];
    __syncthreads();
    return before;
}

// Step 3a, one CTA per query: U = the want-th smallest hi, and the
// candidates (lists with lo <= U) in list order to cand[q * nlist ..] with
// their count in ncand[q]; one work unit (q, first candidate) per 32 of them
// is appended to units. Shared memory: lo and hi bits per list.
__global__ void __launch_bounds__(kSelThreads) route_cand_kernel(const float2* __restrict__ lohi, int nlist,
                                                                 const uint32_t* __restrict__ np_arr, int np_uniform,
                                                                 int* __restrict__ cand, int* __restrict__ ncand,
                                                                 int2* __restrict__ units,
                                                                 uint32_t* __restrict__ nunits) {
    extern __shared__ __align__(16) unsigned char ssm[];
    uint32_t* hi = reinterpret_cast<uint32_t*>(ssm);  // nlist
    float* lo = reinterpret_cast<float*>(hi + nlist);  // nlist
    __shared__ int hist[256];
    __shared__ uint32_t s_p32;
    __shared__ int s_want;
    __shared__ int sm32[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int q = blockIdx.x;
    const int want = min(np_arr ? static_cast<int>(np_arr[q]) : np_uniform, nlist);
    const float2* lq = lohi + static_cast<size_t>(q) * nlist;
    for (int c = tid; c < nlist; c += nt) {
        const float2 v = lq[c];
        lo[c] = v.x;
        hi[c] = __float_as_uint(v.y);  // non-negative: bit order is value order
    }
    const float U = __uint_as_float(block_select<uint32_t>(hi, nlist, want, hist, &s_p32, &s_want));
    int* cq = cand + static_cast<size_t>(q) * nlist;
    int m = 0;
    for (int c0 = 0; c0 < nlist; c0 += nt) {
        const int c = c0 + tid;
        const int flag = (c < nlist && lo[c] <= U) ? 1 : 0;
        int tot = 0;
        const int pos = m + block_scan_flag(flag, sm32, &tot);
        if (flag) cq[pos] = c;
        m += tot;
    }
    if (m < want) {  // only with NaN bounds: every list is a candidate
        __syncthreads();
        for (int c = tid; c < nlist; c += nt) cq[c] = c;
        m = nlist;
    }
    if (tid == 0) {
        ncand[q] = m;
        // the query's exact-key work: one unit per 32 candidates
        const int nu = (m + 31) / 32;
        const uint32_t u0 = atomicAdd(nunits, static_cast<uint32_t>(nu));
        for (int u = 0; u < nu; ++u) units[u0 + u] = make_int2(q, 32 * u);
    }
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Step 3b: exact keys of every unit's (up to) 32 candidates, one warp per
// unit (units dealt round-robin over all warps of the grid). Lane l owns
// candidate jb + l and runs the route GEMM's sequential fp64 FMA chain over
// the dimensions. Per 32-dimension block the warp copies the 32 centroid
// rows' 128-byte pieces (cp.async, 4 bytes per lane per row, coalesced) into
// a padded 32 x 33 tile of a kRkStages ring, kRkStages - 1 blocks ahead; lane
// l reads its row from the tile and the query's values by shuffle.
__global__ void __launch_bounds__(kRkThreads) route_rekey_kernel(
    const int2* __restrict__ units, const uint32_t* __restrict__ nunits, const int* __restrict__ cand,
    const int* __restrict__ ncand, int nlist, int pd, const float* __restrict__ rq, const float* __restrict__ cen,
    const float* __restrict__ qn2, const float* __restrict__ cn2, unsigned long long* __restrict__ ckeys) {
    extern __shared__ __align__(16) float rk_ring[];  // kRkThreads / 32 warps x kRkStages x 32 x 33
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* ring = rk_ring + warp * kRkStages * 32 * 33;
    const uint32_t nu = *nunits;
    const int nb = pd / 32;
    const int gw = blockIdx.x * (kRkThreads / 32) + warp, nw = gridDim.x * (kRkThreads / 32);
    for (uint32_t u = gw; u < nu; u += nw) {
        const int2 un = units[u];
        const int q = un.x, jb = un.y;
        const int nj = min(32, ncand[q] - jb);
        const int* cq = cand + static_cast<size_t>(q) * nlist + jb;
        const int mine = cq[min(lane, nj - 1)];
        const float* qrow = rq + static_cast<size_t>(q) * pd;
        // rows of the unit's candidates (repeating the last one past nj)
        auto issue = [&](int b) {
            float* t = ring + (b % kRkStages) * 32 * 33;
#pragma unroll 8
            for (int j = 0; j < 32; ++j) {
                const int c = __shfl_sync(kFull, mine, j);
                cp_async4(t + j * 33 + lane, cen + static_cast<size_t>(c) * pd + 32 * b + lane);
            }
        };
#pragma unroll
        for (int b = 0; b < kRkStages - 1; ++b) {
            if (b < nb) issue(b);
            cp_async_commit();  // empty groups keep the count uniform
        }
        double acc = 0.0;
        for (int b = 0; b < nb; ++b) {
            if (b + kRkStages - 1 < nb) issue(b + kRkStages - 1);
            cp_async_commit();
            const float qv = qrow[32 * b + lane];
            cp_async_wait<kRkStages - 1>();  // this lane's copies of block b have landed
            __syncwarp();                    // ... and every other lane's
            const float* t = ring + (b % kRkStages) * 32 * 33 + lane * 33;
#pragma unroll
            for (int k = 0; k < 32; ++k)
                acc = __fma_rn(static_cast<double>(__shfl_sync(kFull, qv, k)), static_cast<double>(t[k]), acc);
            __syncwarp();  // the slot is refilled only after every lane has read it
        }
        cp_async_wait<0>();
        if (lane < nj) {
            float d2 = __fmaf_rn(-2.0f, static_cast<float>(acc), __fadd_rn(qn2[q], cn2[mine]));
            if (d2 < 0.0f) d2 = 0.0f;
            ckeys[static_cast<size_t>(q) * nlist + jb + lane] =
                (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) | static_cast<uint32_t>(mine);
        }
    }
}

// Step 3c, one CTA per query: the want smallest exact keys among the
// query's candidates, written in list order with their d2, and the per-list
// pair counts. Shared memory: the candidates' keys.
__global__ void __launch_bounds__(kSelThreads) route_pick_kernel(
    const unsigned long long* __restrict__ ckeys, const int* __restrict__ ncand, int nlist,
    const uint32_t* __restrict__ np_arr, int np_uniform, int np_max, uint32_t* __restrict__ probes,
    float* __restrict__ pd2, uint32_t* __restrict__ list_cnt) {
    extern __shared__ __align__(16) unsigned long long ckey[];  // nlist
    __shared__ int hist[256];
    __shared__ unsigned long long s_p64;
    __shared__ int s_want;
    __shared__ int sm32[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int q = blockIdx.x;
    const int want = min(np_arr ? static_cast<int>(np_arr[q]) : np_uniform, nlist);
    const int m = ncand[q];
    for (int j = tid; j < m; j += nt) ckey[j] = ckeys[static_cast<size_t>(q) * nlist + j];
    const unsigned long long kth = block_select<unsigned long long>(ckey, m, want, hist, &s_p64, &s_want);
    int base = 0;
    for (int j0 = 0; j0 < m; j0 += nt) {
        const int j = j0 + tid;
        const unsigned long long key = j < m ? ckey[j] : ~0ull;
        const int flag = (j < m && key <= kth) ? 1 : 0;
        int tot = 0;
        const int pos = base + block_scan_flag(flag, sm32, &tot);
        if (flag) {
            const uint32_t c = static_cast<uint32_t>(key & 0xFFFFFFFFu);
            const size_t o = static_cast<size_t>(q) * np_max + pos;
            probes[o] = c;
            pd2[o] = __uint_as_float(static_cast<uint32_t>(key >> 32));
            atomicAdd(&list_cnt[c], 1u);
        }
        base += tot;
    }
}

}  // namespace

bool route_tc_applies(const DevIndex& ix, size_t nq) {
    return nq >= kRouteTcMinQueries && ix.nlist <= kRouteTcMaxLists && ix.pd <= kRouteTcMaxDim && ix.pd % kRK == 0;
}

int route_tc(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* np_arr, int np_max,
             cudaStream_t s) {
    const int nlist = ix.nlist, pd = ix.pd;
    const int qrows = static_cast<int>((nq + kRT - 1) / kRT * kRT), crows = (nlist + kRT - 1) / kRT * kRT;
    ws.r_qplane.ensure(static_cast<size_t>(3) * qrows * pd);
    ws.r_cplane.ensure(static_cast<size_t>(3) * crows * pd);
    ws.r_qmeta.ensure(static_cast<size_t>(qrows) * 16);
    ws.r_cmeta.ensure(static_cast<size_t>(crows) * 16);
    ws.ensure_err();
    int launches = 0;
    route_slice_kernel<<<static_cast<unsigned>(qrows / 8), 256, 0, s>>>(
        rq, static_cast<int>(nq), qrows, pd, ws.r_qplane.as<int8_t>(), ws.r_qmeta.as<float4>());
    route_slice_kernel<<<static_cast<unsigned>(crows / 8), 256, 0, s>>>(ix.cen, nlist, crows, pd,
                                                                         ws.r_cplane.as<int8_t>(),
                                                                         ws.r_cmeta.as<float4>());
    launches += 2;
    const CUtensorMap map_q = plane_map(ws.r_qplane.p, static_cast<size_t>(3) * qrows / 8, pd, 16);
    const CUtensorMap map_c = plane_map(ws.r_cplane.p, static_cast<size_t>(3) * crows / 8, pd, 16);
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    const size_t gsmem = static_cast<size_t>(kRStages) * kRStageBytes;
    static bool configured[64] = {};
    if (!configured[dev & 63]) {
        E8QC_CUDA(cudaFuncSetAttribute(route_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(gsmem)));
        configured[dev & 63] = true;
    }
    dim3 g(static_cast<unsigned>(crows / kRT), static_cast<unsigned>(qrows / kRT));
    float2* lohi = ws.b_keys.as<float2>();  // nq x nlist intervals in the key buffer
    route_tc_kernel<<<g, kRThreads, gsmem, s>>>(map_q, map_c, static_cast<int>(nq), nlist, pd, qrows, crows,
                                                 ws.r_qmeta.as<float4>(), ws.r_cmeta.as<float4>(),
                                                 ws.b_qn2.as<float>(), ix.cn2, lohi, ws.err.as<uint32_t>());
    ++launches;
    ws.r_cand.ensure(nq * static_cast<size_t>(nlist) * 4);
    ws.r_ncand.ensure(nq * 4 + 4);  // per query, then the unit count
    ws.r_units.ensure(nq * (static_cast<size_t>(nlist) / 32 + 1) * 8);
    ws.r_ckeys.ensure(nq * static_cast<size_t>(nlist) * 8);
    uint32_t* nunits = reinterpret_cast<uint32_t*>(ws.r_ncand.as<int>() + nq);
    E8QC_CUDA(cudaMemsetAsync(nunits, 0, 4, s));
    const size_t csmem = static_cast<size_t>(nlist) * 8;
    static size_t sconfigured[64] = {};
    if (csmem > 48 * 1024 && sconfigured[dev & 63] < csmem) {
        E8QC_CUDA(cudaFuncSetAttribute(route_cand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(csmem)));
        E8QC_CUDA(cudaFuncSetAttribute(route_pick_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(csmem)));
        sconfigured[dev & 63] = csmem;
    }
    route_cand_kernel<<<static_cast<unsigned>(nq), kSelThreads, csmem, s>>>(
        lohi, nlist, np_arr, np_max, ws.r_cand.as<int>(), ws.r_ncand.as<int>(), ws.r_units.as<int2>(), nunits);
    int sms = 148;
    E8QC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t rksmem = static_cast<size_t>(kRkThreads / 32) * kRkStages * 32 * 33 * 4;
    static bool rkconfigured[64] = {};
    if (!rkconfigured[dev & 63]) {
        E8QC_CUDA(cudaFuncSetAttribute(route_rekey_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(rksmem)));
        rkconfigured[dev & 63] = true;
    }
    route_rekey_kernel<<<static_cast<unsigned>(sms * kRkBlocksPerSm), kRkThreads, rksmem, s>>>(
        ws.r_units.as<int2>(), nunits, ws.r_cand.as<int>(), ws.r_ncand.as<int>(), nlist, pd, rq, ix.cen,
        ws.b_qn2.as<float>(), ix.cn2, ws.r_ckeys.as<unsigned long long>());
    route_pick_kernel<<<static_cast<unsigned>(nq), kSelThreads, csmem, s>>>(
        ws.r_ckeys.as<unsigned long long>(), ws.r_ncand.as<int>(), nlist, np_arr, np_max, np_max,
        ws.b_probes.as<uint32_t>(), ws.b_pd2.as<float>(), ws.b_cnt.as<uint32_t>());
    launches += 3;
    E8QC_CUDA(cudaGetLastError());
    return launches;
}

}  // namespace e8qc
