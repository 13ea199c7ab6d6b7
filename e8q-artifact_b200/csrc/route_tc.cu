// Batch routing keys on the int8 tensor cores, equal to the fp64 route's
// (src/index/ivf_route.cpp:9-27, src/simd/kernels_generic.cpp:13-33: the dot
// accumulated in fp64 in dimension order, d2 = qn2 + cn2 - 2 * float(dot)
// clamped at 0, key = (bits(d2) << 32) | list id).
//
// 1. Slicing (route_slice_kernel): each row x (a rotated query or centroid)
//    is scaled by 127 / 2^e, 2^e > max|x| (exact in fp64: a 24-bit by 7-bit
//    product), and split exactly into seven int8 slices,
//      X = sum_t Q_t 128^-t + rho,  |Q_0| <= 127, |Q_t| <= 64, |rho_i| <= 2^-43,
//    with the row's N = sum_{t>=1} |Q_t| and |X - rho| (rounded up).
// 2. Keys (route_tc_kernel): tcgen05 kind::i8 products of the slices with
//    exact int32 accumulation, the 28 with t + u <= 6 summed by weight w =
//    t + u into seven TMEM accumulators. The epilogue forms the dot in fp64
//    and a rigorous bound on |dot - (the reference's fp64 dot)|: the dropped
//    products (all have t, u >= 1, so at most 2^-49 N_q N_c), the residuals
//    (Cauchy-Schwarz), the fp64 combination, and the reference's own
//    sequential fp64 rounding (n 2^-53 |q||c|, taken twice). When both ends of
//    that interval round to the same float F, float(dot) is F and the key is
//    formed exactly as the reference forms it. Otherwise the pair gets an
//    interval: the key holds a lower bound of its d2 bits with bit 31 of the
//    low word set (list ids stay below 2^31), ub[q * nlist + c] an upper bound
//    (every pair of a row with a NaN or infinite element gets [0, all ones]),
//    and select_kernel computes the exact key of any interval pair that could
//    be selected with route_gemm_kernel's fp64 chain.
// The probes, their d2 and the list counts are the fp64 route's, bit for bit.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "internal.h"
#include "precision.h"
#include "route_tc.h"
#include "tc.cuh"
#include "tma.cuh"
#include "workspace.h"

namespace e8qc {

namespace {

constexpr int kSl = 7;                                 // int8 slices per row
constexpr int kRM = 128;                               // queries per tile (TMEM lanes)
constexpr int kRN = 64;                                // lists per tile
constexpr int kRK = 32;                                // K bytes per chunk (one MMA)
constexpr int kASlab = kRM * kRK;                      // 4 KB: one query slice of one chunk
constexpr int kBSlab = kRN * kRK;                      // 2 KB: one list slice of one chunk
constexpr int kRStageBytes = kSl * (kASlab + kBSlab);  // 42 KB
constexpr int kRStages = 5;
constexpr int kRThreads = 192;
constexpr uint32_t kRCols = 512;  // 7 accumulators x 64 columns, rounded to a power of two
constexpr int kRouteTcMaxLists = 25600;
constexpr int kRouteTcMaxDim = 4096;

// One warp per row of a plane of rows_pad rows (slice t at rows t*rows_pad..):
// rows < n hold src's row, the rest are zero. meta[r] = (2^e, N, |X - rho|,
// 0), or (1, inf, inf, 0) for a row with a NaN or infinite element.
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
    if (mx > 0.0f) (void)frexpf(mx, &e);  // mx < 2^e (an infinite mx is caught per element below)
    const double f = ldexp(127.0, -e);
    double nt[kSl] = {};  // sums of squares of the slices (exact: integers below 2^53)
    double nx = 0.0;
    bool bad = false;
    const size_t slice = static_cast<size_t>(rows_pad) * pd;
    for (int p = lane; p < pd / 16; p += 32) {
        uint32_t w[kSl][4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
#pragma unroll
            for (int t = 0; t < kSl; ++t) w[t][b] = 0u;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int i = p * 16 + b * 4 + k;
                double x = live ? static_cast<double>(row[i]) * f : 0.0;
                if (!(fabs(x) <= 127.0)) {
                    bad = true;
                    x = 0.0;
                }
                double rr = x, xh = 0.0;
#pragma unroll
                for (int t = 0; t < kSl; ++t) {
                    const double qt = rint(rr);      // |qt| <= 127 (t = 0), <= 64 after
                    rr = (rr - qt) * 128.0;          // exact
                    xh += qt * ldexp(1.0, -7 * t);  // exact: 49 significant bits at most
                    nt[t] = __fma_rn(qt, qt, nt[t]);
                    w[t][b] |= static_cast<uint32_t>(static_cast<uint8_t>(static_cast<int8_t>(qt))) << (8 * k);
                }
                nx = __fma_rn(xh, xh, nx);
            }
        }
        const size_t off = tc::il_offset(r, p * 16, pd);
#pragma unroll
        for (int t = 0; t < kSl; ++t)
            *reinterpret_cast<uint4*>(plane + t * slice + off) = make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
    }
    bad = __any_sync(kFull, bad);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int t = 1; t < kSl; ++t) nt[t] += __shfl_xor_sync(kFull, nt[t], o);
        nx += __shfl_xor_sync(kFull, nx, o);
    }
    if (lane == 0) {
        const float inf = __int_as_float(0x7f800000);
        double N = 0.0;
#pragma unroll
        for (int t = 1; t < kSl; ++t) N = __dadd_ru(N, __dsqrt_ru(nt[t]));
        // nx carries a few ulps of rounding: 2^-40 of slack, then round up
        meta[r] = bad ? make_float4(1.0f, inf, inf, 0.0f)
                      : make_float4(ldexpf(1.0f, e), __double2float_ru(N),
                                    __double2float_ru(__dsqrt_ru(nx * (1.0 + 0x1p-40))), 0.0f);
    }
}

// One 128-query x 64-list tile per CTA. Warp 0 loads the fourteen slices of
// each 32-byte K-chunk by TMA into a kRStages ring, one thread of warp 1
// issues the chunk's 28 kind::i8 MMAs, warps 2-5 read the seven
// accumulators (thread = query row) and write the keys. Waits are bounded; a
// timeout sets the error word.
__global__ void __launch_bounds__(kRThreads, 1) route_tc_kernel(
    const __grid_constant__ CUtensorMap map_q, const __grid_constant__ CUtensorMap map_c, int nq, int nlist, int pd,
    int qrows_pad, int crows_pad, const float4* __restrict__ qmeta, const float4* __restrict__ cmeta,
    const float* __restrict__ qn2, const float* __restrict__ cn2, unsigned long long* __restrict__ keys,
    uint32_t* __restrict__ ub, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char rsm[];
    __shared__ __align__(8) uint64_t full[kRStages], empty[kRStages], tfull, fin;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ double s_cs[kRN];  // the list's 2^e / 127^2
    __shared__ double s_cr[kRN];  // sqrt(cn2), rounded up
    __shared__ float s_cN[kRN], s_cX[kRN], s_cn2[kRN];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nK = pd / kRK;
    const int q0 = blockIdx.y * kRM, c0 = blockIdx.x * kRN;
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
    for (int j = tid; j < kRN; j += blockDim.x) {
        const int c = c0 + j;
        const float4 cm = c < nlist ? cmeta[c] : make_float4(1.0f, 0.0f, 0.0f, 0.0f);
        const float cc = c < nlist ? cn2[c] : 0.0f;
        s_cs[j] = static_cast<double>(cm.x) / 16129.0;
        s_cN[j] = cm.y;
        s_cX[j] = cm.z;
        s_cn2[j] = cc;
        s_cr[j] = __dsqrt_ru(fmax(static_cast<double>(cc), 0.0));
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
                // 16 (queries) / 8 (lists) row groups x 8 * kRK bytes (2 * kRK u32 at x = kc * 2 * kRK)
#pragma unroll
                for (int t = 0; t < kSl; ++t) {
                    tma_load_2d(base + t * kASlab, &map_q, kc * 2 * kRK, (t * qrows_pad + q0) >> 3, &full[st]);
                    tma_load_2d(base + kSl * kASlab + t * kBSlab, &map_c, kc * 2 * kRK, (t * crows_pad + c0) >> 3,
                                &full[st]);
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
            const uint32_t idesc = tc::idesc_i8(kRM, kRN);
            const uint32_t sbo = (kRK / 16) * 128u;
            bool issued = false;
            for (int kc = 0; kc < nK && !s_abort; ++kc) {
                const int st = kc % kRStages;
                if (!mbar_wait_or_abort(&full[st], (kc / kRStages) & 1u, &s_abort)) break;
                tc::fence_after_sync();
                const uint32_t a0 = tc::saddr(rsm + st * kRStageBytes), b0 = a0 + kSl * kASlab;
#pragma unroll
                for (int s2 = 0; s2 < kRK / 32; ++s2) {
                    const uint32_t first = (kc > 0 || s2 > 0) ? 1u : 0u;
#pragma unroll
                    for (int w = 0; w < kSl; ++w)
#pragma unroll
                        for (int t = 0; t <= w; ++t)
                            tc::mma_i8(tmem + static_cast<uint32_t>(w * kRN),
                                       tc::smem_desc(a0 + t * kASlab + 256u * s2, 128u, sbo),
                                       tc::smem_desc(b0 + (w - t) * kBSlab + 256u * s2, 128u, sbo), idesc,
                                       t == 0 ? first : 1u);
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
        const float qqf = q < nq ? qn2[q] : 0.0f;
        const double qr = __dsqrt_ru(fmax(static_cast<double>(qqf), 0.0));
        const double n = static_cast<double>(pd), rn = sqrt(n);
        if (mbar_wait_or_abort(&tfull, 0u, &s_abort)) {
            tc::fence_after_sync();
            for (int cb = 0; cb < kRN; cb += 8) {
                uint32_t acc[kSl][8];
#pragma unroll
                for (int w = 0; w < kSl; ++w)
                    tc::tmem_ld8(tmem + ((static_cast<uint32_t>(q4) * 32u) << 16) + w * kRN + cb, acc[w]);
                tc::tmem_ld_wait();
                if (q >= nq) continue;
                unsigned long long* krow = keys + static_cast<size_t>(q) * nlist + c0 + cb;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int c = c0 + cb + j;
                    if (c >= nlist) continue;
                    double S = 0.0;
#pragma unroll
                    for (int w = kSl - 1; w >= 0; --w)
                        S = __fma_rn(static_cast<double>(static_cast<int>(acc[w][j])), ldexp(1.0, -7 * w), S);
                    const double sc = static_cast<double>(qm.x) * s_cs[cb + j];
                    const double dot = S * sc;
                    // |sum x y - S| over the scaled rows: dropped products + residuals
                    const double E = 0x1p-49 * static_cast<double>(qm.y) * s_cN[cb + j] +
                                     0x1p-43 * rn * (static_cast<double>(qm.z) + s_cX[cb + j]) + n * 0x1p-86;
                    const double er =
                        E * sc * (1.0 + 0x1p-40) + fabs(dot) * 0x1p-48 + n * 0x1p-52 * qr * s_cr[cb + j];
                    const float s2 = __fadd_rn(qqf, s_cn2[cb + j]);
                    unsigned long long key;
                    if (er <= 1e300) {
                        // float(reference dot) lies in [Flo, Fhi]; d2 = fma(-2, F, s2) falls as F grows
                        const float Flo = __double2float_rn(dot - er), Fhi = __double2float_rn(dot + er);
                        const float lo = fmaxf(__fmaf_rn(-2.0f, Fhi, s2), 0.0f);
                        if (Flo == Fhi) {
                            key = (static_cast<unsigned long long>(__float_as_uint(lo)) << 32) | static_cast<uint32_t>(c);
                        } else {
                            key = (static_cast<unsigned long long>(__float_as_uint(lo)) << 32) | 0x80000000ull |
                                  static_cast<uint32_t>(c);
                            ub[static_cast<size_t>(q) * nlist + c] = __float_as_uint(fmaxf(__fmaf_rn(-2.0f, Flo, s2), 0.0f));
                        }
                    } else {  // a NaN or infinite input: any d2 (NaN bits included)
                        key = 0x80000000ull | static_cast<uint32_t>(c);
                        ub[static_cast<size_t>(q) * nlist + c] = 0xFFFFFFFFu;
                    }
                    krow[j] = key;
                }
            }
        }
    }
    __syncthreads();
    if (s_abort && tid == 0) atomicOr(err, kErrWaitTimeout);
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem, kRCols);
}

}  // namespace

bool route_tc_applies(const DevIndex& ix, size_t nq) {
    return nq >= kRouteTcMinQueries && ix.nlist <= kRouteTcMaxLists && ix.pd <= kRouteTcMaxDim && ix.pd % kRK == 0;
}

int route_tc_keys(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, cudaStream_t s) {
    const int nlist = ix.nlist, pd = ix.pd;
    const int qrows = static_cast<int>((nq + kRM - 1) / kRM * kRM), crows = (nlist + kRN - 1) / kRN * kRN;
    ws.r_qplane.ensure(static_cast<size_t>(kSl) * qrows * pd);
    ws.r_cplane.ensure(static_cast<size_t>(kSl) * crows * pd);
    ws.r_qmeta.ensure(static_cast<size_t>(qrows) * 16);
    ws.r_cmeta.ensure(static_cast<size_t>(crows) * 16);
    ws.r_ub.ensure(nq * static_cast<size_t>(nlist) * 4);
    ws.ensure_err();
    route_slice_kernel<<<static_cast<unsigned>(qrows / 8), 256, 0, s>>>(
        rq, static_cast<int>(nq), qrows, pd, ws.r_qplane.as<int8_t>(), ws.r_qmeta.as<float4>());
    route_slice_kernel<<<static_cast<unsigned>(crows / 8), 256, 0, s>>>(ix.cen, nlist, crows, pd,
                                                                         ws.r_cplane.as<int8_t>(),
                                                                         ws.r_cmeta.as<float4>());
    const CUtensorMap map_q = plane_map(ws.r_qplane.p, static_cast<size_t>(kSl) * qrows / 8, pd, kRM / 8, 2 * kRK);
    const CUtensorMap map_c = plane_map(ws.r_cplane.p, static_cast<size_t>(kSl) * crows / 8, pd, kRN / 8, 2 * kRK);
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    const size_t gsmem = static_cast<size_t>(kRStages) * kRStageBytes;
    static bool configured[64] = {};
    if (!configured[dev & 63]) {
        E8QC_CUDA(cudaFuncSetAttribute(route_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(gsmem)));
        configured[dev & 63] = true;
    }
    dim3 g(static_cast<unsigned>(crows / kRN), static_cast<unsigned>(qrows / kRM));
    route_tc_kernel<<<g, kRThreads, gsmem, s>>>(map_q, map_c, static_cast<int>(nq), nlist, pd, qrows, crows,
                                                 ws.r_qmeta.as<float4>(), ws.r_cmeta.as<float4>(),
                                                 ws.b_qn2.as<float>(), ix.cn2, ws.b_keys.as<unsigned long long>(),
                                                 ws.r_ub.as<uint32_t>(), ws.err.as<uint32_t>());
    E8QC_CUDA(cudaGetLastError());
    return 3;
}

}  // namespace e8qc
