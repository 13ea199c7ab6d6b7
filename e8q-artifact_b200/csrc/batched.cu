// Batched search: many queries share each list's decode.
//
//   1. qn2 + route GEMM: d2[q][c] = |q|^2 + |c|^2 - 2 q.c (fp32 products summed
//      in fp64, the plain path's arithmetic), packed (d2 bits << 32 | c) keys.
//   2. per-query top-nprobe select (radix select, as in the plain path).
//   3. group the (query, list) pairs by list; cut each list's pairs into work
//      items of up to QT queries.
//   4. persistent scan: CTAs pull items off a device queue. For an item the
//      CTA decodes the list's codes 64 dimensions at a time into shared memory
//      (levels, fp32) and runs a register-tiled QT x VT fp32 contraction with
//      the item's queries; the epilogue forms the exact estimator
//      (d2 + h3) - 2*g1*S and updates each query's top-k in shared memory.
//      Every (query, vector) score accumulates over the dimensions in the same
//      fixed order whatever else is in the batch, so results do not depend on
//      batch composition.
//   5. per-query merge of its nprobe partial lists.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "device_common.cuh"
#include "internal.h"
#include "me8q.h"
#include "route_tc.h"
#include "workspace.h"

namespace e8qc {

namespace {

__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

constexpr int kBT = 256;   // threads of the scan kernel
constexpr int kQT = 64;    // queries per work item
constexpr int kVT = 128;   // vectors per inner tile (4 code tiles)
constexpr int kKC = 64;    // dimensions per decode chunk (8 blocks)

// |q|^2 with the plain path's reduction order (route_one_kernel): 256 threads
// strided, warp xor tree, warps summed in order.
__global__ void qn2_kernel(const float* __restrict__ rq, int pd, float* __restrict__ qn2) {
    __shared__ double red[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float* q = rq + static_cast<size_t>(blockIdx.x) * pd;
    double part = 0.0;
    for (int i = tid; i < pd; i += 256) {
        const float v = q[i];
        part += static_cast<double>(v) * static_cast<double>(v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    if (lane == 0) red[warp] = part;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int i = 0; i < 8; ++i) s += red[i];
        qn2[blockIdx.x] = static_cast<float>(s);
    }
}

// Route GEMM: 128 queries x 64 centroids per CTA of 128 threads, 8 x 8 fp64
// accumulators per thread (queries ty*4+i and 64+ty*4+i, centroids tx*4+j and
// 32+tx*4+j). 16-dim chunks of both operands are converted to fp64 once, when
// they are staged (transposed) in shared memory; the next chunk is fetched into
// registers while the current one is multiplied. Every (query, list) dot is one
// fp64 FMA chain over the dimensions in order (products of two floats are exact
// in fp64), so the result does not depend on the tiling.
constexpr int kRouteBQ = 128, kRouteBC = 64, kRouteBK = 16;
__global__ void __launch_bounds__(128, 2) route_gemm_kernel(const float* __restrict__ rq, int nq,
                                                            const float* __restrict__ cen,
                                                            const float* __restrict__ cn2, int nlist, int pd,
                                                            const float* __restrict__ qn2,
                                                            uint64_t* __restrict__ keys) {
    __shared__ __align__(16) double As[kRouteBK][kRouteBQ + 2];
    __shared__ __align__(16) double Bs[kRouteBK][kRouteBC + 2];
    const int tid = threadIdx.x;
    const int q0 = blockIdx.y * kRouteBQ, c0 = blockIdx.x * kRouteBC;
    const int ty = tid >> 3, tx = tid & 7;
    // staging: A chunk = 128 rows x 4 float4 (4 per thread), B = 64 x 4 (2 per thread)
    float4 ra[4], rb[2];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int e = tid + h * 128, r = e >> 2, k4 = (e & 3) * 4;
            ra[h] = q0 + r < nq ? *reinterpret_cast<const float4*>(rq + static_cast<size_t>(q0 + r) * pd + k0 + k4)
                                : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int e = tid + h * 128, r = e >> 2, k4 = (e & 3) * 4;
            rb[h] = c0 + r < nlist ? *reinterpret_cast<const float4*>(cen + static_cast<size_t>(c0 + r) * pd + k0 + k4)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    auto stage = [&]() {
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int e = tid + h * 128, r = e >> 2, k4 = (e & 3) * 4;
            As[k4 + 0][r] = ra[h].x;
            As[k4 + 1][r] = ra[h].y;
            As[k4 + 2][r] = ra[h].z;
            As[k4 + 3][r] = ra[h].w;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int e = tid + h * 128, r = e >> 2, k4 = (e & 3) * 4;
            Bs[k4 + 0][r] = rb[h].x;
            Bs[k4 + 1][r] = rb[h].y;
            Bs[k4 + 2][r] = rb[h].z;
            Bs[k4 + 3][r] = rb[h].w;
        }
    };
    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    fetch(0);
    for (int k0 = 0; k0 < pd; k0 += kRouteBK) {
        stage();
        __syncthreads();
        if (k0 + kRouteBK < pd) fetch(k0 + kRouteBK);
#pragma unroll
        for (int kk = 0; kk < kRouteBK; ++kk) {
            double a[8], b[8];
            const double2* ar = reinterpret_cast<const double2*>(&As[kk][0]);
            const double2* br = reinterpret_cast<const double2*>(&Bs[kk][0]);
            const double2 a0 = ar[ty * 2], a1 = ar[ty * 2 + 1], a2 = ar[32 + ty * 2], a3 = ar[32 + ty * 2 + 1];
            const double2 b0 = br[tx * 2], b1 = br[tx * 2 + 1], b2 = br[16 + tx * 2], b3 = br[16 + tx * 2 + 1];
            a[0] = a0.x, a[1] = a0.y, a[2] = a1.x, a[3] = a1.y, a[4] = a2.x, a[5] = a2.y, a[6] = a3.x, a[7] = a3.y;
            b[0] = b0.x, b[1] = b0.y, b[2] = b1.x, b[3] = b1.y, b[4] = b2.x, b[5] = b2.y, b[6] = b3.x, b[7] = b3.y;
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = __fma_rn(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int qi = q0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
        if (qi >= nq) continue;
        const float qq = qn2[qi];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int ci = c0 + (j < 4 ? tx * 4 + j : 32 + tx * 4 + (j - 4));
            if (ci >= nlist) continue;
            float d2 = __fmaf_rn(-2.0f, static_cast<float>(acc[i][j]), __fadd_rn(qq, cn2[ci]));
            if (d2 < 0.0f) d2 = 0.0f;
            keys[static_cast<size_t>(qi) * nlist + ci] =
                (static_cast<uint64_t>(__float_as_uint(d2)) << 32) | static_cast<uint32_t>(ci);
        }
    }
}

// The want-th smallest of n 32-bit values in shared memory by MSB radix
// select with 8-bit digits (four passes); every thread of the block gets it.
// hist: 256 ints; sm: 2 ints.
__device__ uint32_t block_select32(const uint32_t* v, int n, int want, int* hist, int* sm) {
    const int tid = threadIdx.x, nt = blockDim.x;
    uint32_t prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = tid; i < 256; i += nt) hist[i] = 0;
        __syncthreads();
        for (int c = tid; c < n; c += nt) {
            const uint32_t x = v[c];
            if ((x & mask) == prefix) atomicAdd(&hist[(x >> shift) & 255u], 1);
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
            const unsigned hit = __ballot_sync(kFull, excl < want && incl >= want);
            const int owner = __ffs(hit) - 1;
            if (tid == owner) {
                int cum = excl, sel = 0;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    if (cum + cnt[j] >= want) {
                        sel = j;
                        break;
                    }
                    cum += cnt[j];
                }
                sm[0] = tid * 8 + sel;
                sm[1] = want - cum;
            }
        }
        __syncthreads();
        prefix |= static_cast<uint32_t>(sm[0]) << shift;
        mask |= 0xFFu << shift;
        want = sm[1];
        __syncthreads();
    }
    return prefix;
}

// d2 bits of (query row qr, list c) by route_gemm_kernel's sequential fp64
// chain, computed by a whole warp: per 32-dimension block each lane loads
// one element of both rows (coalesced, the next block in flight) and every
// lane runs the same chain on the shuffled values.
__device__ uint32_t warp_exact_d2(const float* __restrict__ qr, const float* __restrict__ cen, int pd, float qq,
                                  float cc, int c) {
    const int lane = threadIdx.x & 31;
    const float* cr = cen + static_cast<size_t>(c) * pd;
    float qv = qr[lane], cv = cr[lane];
    double acc = 0.0;
    for (int k = 0; k < pd; k += 32) {
        const float nq = k + 32 < pd ? qr[k + 32 + lane] : 0.0f;
        const float nc = k + 32 < pd ? cr[k + 32 + lane] : 0.0f;
#pragma unroll
        for (int l = 0; l < 32; ++l)
            acc = __fma_rn(static_cast<double>(__shfl_sync(kFull, qv, l)), static_cast<double>(__shfl_sync(kFull, cv, l)),
                           acc);
        qv = nq;
        cv = nc;
    }
    float d2 = __fmaf_rn(-2.0f, static_cast<float>(acc), __fadd_rn(qq, cc));
    if (d2 < 0.0f) d2 = 0.0f;
    return __float_as_uint(d2);
}

// Per-query top-nprobe: one CTA per query. A key is exact, or (from the
// tensor-core route) an interval: the low word's bit 31 set, the high word a
// lower bound of the list's d2 bits and ub[q * nlist + c] an upper bound. The
// nprobe-th smallest upper bound U bounds the true nprobe-th d2; interval
// lists whose lower bound is at most U get their exact key (the fp64 chain),
// the rest keep their lower bound (above U, never selected). Then the
// nprobe-th smallest d2 T (U itself when nothing was resolved; 8-bit radix
// select), and the lists with d2 < T
// plus the first ones in list order with d2 == T -- the nprobe smallest
// 64-bit keys -- are written in list order with their d2.
__global__ void select_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ ub, int nlist,
                              const uint32_t* __restrict__ np_arr, int np_uniform, int np_max,
                              const float* __restrict__ rq, const float* __restrict__ cen, int pd,
                              const float* __restrict__ qn2, const float* __restrict__ cn2,
                              uint32_t* __restrict__ probes, float* __restrict__ pd2,
                              uint32_t* __restrict__ list_cnt) {
    extern __shared__ uint32_t shi[];  // nlist d2 words, then nlist interval lower bounds
    uint32_t* slb = shi + nlist;
    __shared__ int hist[256];
    __shared__ int sm[34];
    __shared__ int s_any, s_nres;
    __shared__ int s_res[256];  // interval lists to resolve (more are resolved in further rounds)
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int q = blockIdx.x;
    const int want = min(np_arr ? static_cast<int>(np_arr[q]) : np_uniform, nlist);
    const unsigned long long* kq = reinterpret_cast<const unsigned long long*>(keys) + static_cast<size_t>(q) * nlist;
    if (tid == 0) s_any = 0;
    __syncthreads();
    bool any = false;
    for (int c = tid; c < nlist; c += nt) {
        const unsigned long long key = kq[c];
        if (key & 0x80000000ull) {
            slb[c] = static_cast<uint32_t>(key >> 32);
            shi[c] = ub[static_cast<size_t>(q) * nlist + c];
            any = true;
        } else {
            slb[c] = 0xFFFFFFFFu;  // exact
            shi[c] = static_cast<uint32_t>(key >> 32);
        }
    }
    if (any) s_any = 1;
    __syncthreads();
    uint32_t T = 0;
    bool have_T = false;
    if (s_any) {
        const uint32_t U = block_select32(shi, nlist, want, hist, sm);
        int resolved = 0;
        const float* qr = rq + static_cast<size_t>(q) * pd;
        // interval lists that could be selected get their exact d2 (one warp
        // each); the others keep their lower bound, above U
        for (int c0 = 0; c0 < nlist; c0 += 256) {
            if (tid == 0) s_nres = 0;
            __syncthreads();
            for (int c = c0 + tid; c < min(nlist, c0 + 256); c += nt) {
                if (slb[c] == 0xFFFFFFFFu) continue;
                if (slb[c] <= U) s_res[atomicAdd(&s_nres, 1)] = c;
                else shi[c] = slb[c];
            }
            __syncthreads();
            resolved += s_nres;
            for (int i = warp; i < s_nres; i += nw) {
                const int c = s_res[i];
                const uint32_t d = warp_exact_d2(qr, cen, pd, qn2[q], cn2[c], c);
                if (lane == 0) shi[c] = d;
            }
            __syncthreads();
        }
        // nothing resolved: every interval list now sits above U, which stays
        // the want-th smallest value
        if (resolved == 0) {
            T = U;
            have_T = true;
        }
    }
    if (!have_T) T = block_select32(shi, nlist, want, hist, sm);
    // lists below T, then ties at T in list order, up to want
    int below = 0;
    for (int c0 = 0; c0 < nlist; c0 += nt) {
        const int c = c0 + tid;
        const int f = (c < nlist && shi[c] < T) ? 1 : 0;
        below += __syncthreads_count(f);
    }
    int base = 0, ties = 0;
    const int room = want - below;  // ties taken
    for (int c0 = 0; c0 < nlist; c0 += nt) {
        const int c = c0 + tid;
        const uint32_t h = c < nlist ? shi[c] : 0xFFFFFFFFu;
        const int tie = (c < nlist && h == T) ? 1 : 0;
        // block exclusive scans of (tie) and of (selected)
        int x = tie;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sm[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int v = lane < nw ? sm[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, v, o);
                if (lane >= o) v += y;
            }
            sm[lane] = v;
        }
        __syncthreads();
        const int tie_rank = ties + (warp > 0 ? sm[warp - 1] : 0) + x - tie;
        const int tie_tot = sm[nw - 1];
        __syncthreads();
        const int flag = (c < nlist && (h < T || (tie && tie_rank < room))) ? 1 : 0;
        x = flag;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sm[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int v = lane < nw ? sm[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, v, o);
                if (lane >= o) v += y;
            }
            sm[lane] = v;
        }
        __syncthreads();
        const int pos = base + (warp > 0 ? sm[warp - 1] : 0) + x - flag;
        const int tot = sm[nw - 1];
        __syncthreads();
        if (flag) {
            const size_t o = static_cast<size_t>(q) * np_max + pos;
            probes[o] = static_cast<uint32_t>(c);
            pd2[o] = __uint_as_float(h);
            atomicAdd(&list_cnt[c], 1u);
        }
        base += tot;
        ties += tie_tot;
    }
}

// Items: list order `order`, per list ceil(cnt / qt) items. One CTA scans the
// lists (nlist is small) and writes pair offsets and item descriptors.
__global__ void items_kernel(const uint32_t* __restrict__ list_cnt, const uint32_t* __restrict__ order,
                             int nlist, uint32_t* __restrict__ pair_off, uint32_t* __restrict__ fill,
                             uint4* __restrict__ items, uint32_t* __restrict__ n_items, int item_cap, uint32_t qt,
                             uint32_t align) {
    __shared__ uint32_t s_pairs, s_items;
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    if (tid == 0) {
        s_pairs = 0;
        s_items = 0;
    }
    __syncthreads();
    for (int i0 = 0; i0 < nlist; i0 += nt) {
        const int i = i0 + tid;
        const uint32_t L = i < nlist ? order[i] : 0;
        const uint32_t cnt = i < nlist ? list_cnt[L] : 0;
        const uint32_t cpad = (cnt + align - 1) / align * align;  // each list's pairs start aligned
        const uint32_t nit = (cnt + qt - 1) / qt;
        // two block scans (pairs, items)
        uint32_t xp = cpad, xi = nit;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t yp = __shfl_up_sync(kFull, xp, o), yi = __shfl_up_sync(kFull, xi, o);
            if (lane >= o) {
                xp += yp;
                xi += yi;
            }
        }
        __shared__ uint32_t wp[32], wi[32];
        if (lane == 31) {
            wp[warp] = xp;
            wi[warp] = xi;
        }
        __syncthreads();
        if (warp == 0) {
            uint32_t sp = lane < nw ? wp[lane] : 0, si = lane < nw ? wi[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t yp = __shfl_up_sync(kFull, sp, o), yi = __shfl_up_sync(kFull, si, o);
                if (lane >= o) {
                    sp += yp;
                    si += yi;
                }
            }
            wp[lane] = sp;
            wi[lane] = si;
        }
        __syncthreads();
        const uint32_t pbase = s_pairs + (warp > 0 ? wp[warp - 1] : 0) + xp - cpad;
        const uint32_t ibase = s_items + (warp > 0 ? wi[warp - 1] : 0) + xi - nit;
        if (i < nlist) {
            pair_off[L] = pbase;
            fill[L] = 0;
            for (uint32_t t = 0; t < nit; ++t) {
                const uint32_t idx = ibase + t;
                if (static_cast<int>(idx) < item_cap)
                    items[idx] = make_uint4(L, pbase + t * qt, min(qt, cnt - t * qt), t);  // w: item index within its list
            }
        }
        __syncthreads();
        if (tid == 0) {
            s_pairs += wp[nw - 1];
            s_items += wi[nw - 1];
        }
        __syncthreads();
    }
    if (tid == 0) *n_items = min(s_items, static_cast<uint32_t>(item_cap));
}

// Scatter each (query, probe) pair into its list's pair range.
__global__ void scatter_kernel(const uint32_t* __restrict__ probes, const float* __restrict__ pd2, int nq,
                               const uint32_t* __restrict__ np_arr, int np_uniform, int np_max,
                               const uint32_t* __restrict__ pair_off, uint32_t* __restrict__ fill,
                               uint32_t* __restrict__ pair_q, float* __restrict__ pair_d2,
                               uint32_t* __restrict__ pos_of) {
    const size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<size_t>(nq) * np_max) return;
    const int q = static_cast<int>(e / np_max), j = static_cast<int>(e % np_max);
    const int np = np_arr ? static_cast<int>(np_arr[q]) : np_uniform;
    if (j >= np) return;
    const uint32_t L = probes[e];
    const uint32_t pos = pair_off[L] + atomicAdd(&fill[L], 1u);
    pair_q[pos] = static_cast<uint32_t>(q);
    pair_d2[pos] = pd2[e];
    pos_of[e] = pos;
}

// Word `w` of the code stream of the vector in lane `lane` of tile `gt`.
__device__ __forceinline__ uint32_t code_word(const DevIndex& ix, uint32_t gt, int lane, int w) {
    const uint32_t* base = reinterpret_cast<const uint32_t*>(ix.codes + (static_cast<size_t>(gt) * ix.nch + (w >> 2)) * 32 + lane);
    return __ldg(base + (w & 3));
}

// Persistent scan over work items (see file comment).
//   shared: Qs[2][kKC][kQT], Ls[2][kKC][kVT], table[2*Q], top-k [kQT][k_max]
template <int BITS>
__global__ void __launch_bounds__(kBT) batched_scan_kernel(
    DevIndex ix, const float* __restrict__ rq, const uint4* __restrict__ items, const uint32_t* __restrict__ n_items,
    uint32_t* __restrict__ head, const uint32_t* __restrict__ pair_q, const float* __restrict__ pair_d2,
    const uint32_t* __restrict__ k_arr, int k_uniform, int k_max, float* __restrict__ part_d,
    uint32_t* __restrict__ part_id, unsigned long long* __restrict__ cand_count) {
    extern __shared__ __align__(16) float bsm[];
    constexpr int Q = 1 << BITS;
    float* Qs = bsm;                                  // 2 * kKC * kQT
    float* Ls = Qs + 2 * kKC * kQT;                   // 2 * kKC * kVT
    float* tab = Ls + 2 * kKC * kVT;                  // 2 * Q
    float* tk_d = tab + 2 * Q;                        // kQT * k_max
    uint32_t* tk_i = reinterpret_cast<uint32_t*>(tk_d + kQT * k_max);
    __shared__ uint4 s_item;
    __shared__ uint32_t s_q[kQT];
    __shared__ float s_d2[kQT];
    __shared__ int s_k[kQT];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int pd = ix.pd;
    constexpr int bits = BITS;
    for (int e = tid; e < 2 * Q; e += kBT) tab[e] = ix.tab[e];
    const int nK = pd / kKC;  // pd is a multiple of 64
    const int tq = tid >> 4, tv = tid & 15;
    const uint32_t NI = *n_items;
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
        if (tid < kQT) {
            const bool ok = tid < m;
            const uint32_t qq = ok ? pair_q[pbase + tid] : 0u;
            s_q[tid] = qq;
            s_d2[tid] = ok ? pair_d2[pbase + tid] : 0.0f;
            s_k[tid] = ok ? (k_arr ? static_cast<int>(k_arr[qq]) : k_uniform) : 0;
        }
        for (int e = tid; e < kQT * k_max; e += kBT) {
            tk_d[e] = inf_f();
            tk_i[e] = 0xFFFFFFFFu;
        }
        __syncthreads();
        const uint32_t len = ix.list_len[L];
        const uint32_t tile0 = ix.tile_begin[L];
        if (tid == 0) {
            atomicAdd(cand_count, static_cast<unsigned long long>(len) * m);  // (query, vector) pairs
            atomicAdd(cand_count + 1, static_cast<unsigned long long>(len));  // vectors read
            if (item.w == 0) atomicAdd(cand_count + 2, static_cast<unsigned long long>(len));  // once per list
        }
        for (uint32_t v0 = 0; v0 < len; v0 += kVT) {
            float acc[4][8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
            for (int kc = 0; kc < nK; ++kc) {
                float* Qb = Qs + (kc & 1) * kKC * kQT;
                float* Lb = Ls + (kc & 1) * kKC * kVT;
                // stage queries: Qb[kk][q]
                {
                    const int q = tid & 63, part = tid >> 6;  // 4 parts x 16 dims
                    const float* src = rq + static_cast<size_t>(s_q[q]) * pd + kc * kKC + part * 16;
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const float4 v = q < m ? *reinterpret_cast<const float4*>(src + 4 * r)
                                               : make_float4(0.f, 0.f, 0.f, 0.f);
                        const int kk = part * 16 + 4 * r;
                        Qb[(kk + 0) * kQT + q] = v.x;
                        Qb[(kk + 1) * kQT + q] = v.y;
                        Qb[(kk + 2) * kQT + q] = v.z;
                        Qb[(kk + 3) * kQT + q] = v.w;
                    }
                }
                // decode levels: thread -> (vector v, half h): blocks 8kc+4h .. +4
                {
                    const int v = tid & 127, h = tid >> 7;
                    const uint32_t vi = v0 + v;
                    const bool live = vi < len;
                    const uint32_t gt = tile0 + (vi >> 5);
                    const int vl = static_cast<int>(vi & 31);
                    const int w0 = bits * (2 * kc + h);  // first word of the 4 blocks
                    uint32_t w[BITS + 1];
#pragma unroll
                    for (int j = 0; j < BITS; ++j) w[j] = live ? code_word(ix, gt, vl, w0 + j) : 0u;
                    w[BITS] = 0u;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        uint32_t par = 0, dg[8];
                        const int base = b * 8 * bits;
#pragma unroll
                        for (int i = 0; i < 7; ++i) {
                            dg[i] = field(w, base + i * bits, bits);
                            par ^= dg[i];
                        }
                        const uint32_t f7 = field(w, base + 7 * bits, bits);
                        dg[7] = (f7 & ~1u) | (par & 1u);
                        const int br = static_cast<int>(f7 & 1u);
                        const float* t = tab + br * Q;
                        const int kk0 = h * 32 + b * 8;
#pragma unroll
                        for (int i = 0; i < 8; ++i) Lb[(kk0 + i) * kVT + v] = live ? t[dg[i]] : 0.0f;
                    }
                }
                __syncthreads();
#pragma unroll 4
                for (int kk = 0; kk < kKC; ++kk) {
                    const float4 a = *reinterpret_cast<const float4*>(Qb + kk * kQT + tq * 4);
                    const float4 b0 = *reinterpret_cast<const float4*>(Lb + kk * kVT + tv * 4);
                    const float4 b1 = *reinterpret_cast<const float4*>(Lb + kk * kVT + 64 + tv * 4);
                    const float av[4] = {a.x, a.y, a.z, a.w};
                    const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[i][j] = __fmaf_rn(av[i], bv[j], acc[i][j]);
                }
            }
            __syncthreads();
            // epilogue: distances to shared memory (reuse Ls), then per-query top-k
            float* D = Ls;  // kQT x kVT
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int vv = j < 4 ? tv * 4 + j : 64 + tv * 4 + (j - 4);
                const uint32_t vi = v0 + vv;
                const bool live = vi < len;
                const size_t slot = static_cast<size_t>(tile0 + (vi >> 5)) * 32 + (vi & 31);
                const float g1 = live ? __ldg(ix.g1 + slot) : 0.0f;
                const float h3 = live ? __ldg(ix.h3 + slot) : 0.0f;
                const float m2g = -__fmul_rn(2.0f, g1);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int q = tq * 4 + i;
                    D[q * kVT + vv] = live ? __fmaf_rn(m2g, acc[i][j], __fadd_rn(s_d2[q], h3)) : inf_f();
                }
            }
            __syncthreads();
            for (int q = warp; q < m; q += kBT / 32) {
                const int kq = s_k[q];
                WarpTopK top;
                top.init(kq);
                // load the query's current list
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const int j = s * 32 + lane;
                    if (j < kq) {
                        top.d[s] = tk_d[q * k_max + j];
                        top.id[s] = tk_i[q * k_max + j];
                    }
                }
                top.refresh_threshold();
                for (int c = 0; c < kVT; c += 32) {
                    const uint32_t vi = v0 + c + lane;
                    const bool live = vi < len;
                    const float dist = D[q * kVT + c + lane];
                    const size_t slot = static_cast<size_t>(tile0 + (vi >> 5)) * 32 + (vi & 31);
                    top.offer(dist, live, [&] { return __ldg(ix.ids + slot); });
                }
                top.store(tk_d + q * k_max, tk_i + q * k_max, kq);
            }
            __syncthreads();
        }
        // write the item's per-pair lists
        for (int e = tid; e < m * k_max; e += kBT) {
            const int q = e / k_max, j = e - q * k_max;
            const size_t o = static_cast<size_t>(pbase + q) * k_max + j;
            part_d[o] = tk_d[q * k_max + j];
            part_id[o] = tk_i[q * k_max + j];
        }
    }
}

// ME8Q: half of a 64-dim chunk (4 blocks, 32 dims) of one vector at rate B,
// decoded to levels scaled by the vector's coef for the chunk's run.
template <int B>
__device__ __forceinline__ void me8q_decode_half(const DevIndex& ix, uint32_t gt, int vl, bool live, int w0,
                                                 const float* __restrict__ lev, float cf, float* Lb, int kk0,
                                                 int v) {
    uint32_t w[B + 1];
#pragma unroll
    for (int j = 0; j < B; ++j) w[j] = live ? code_word(ix, gt, vl, w0 + j) : 0u;
    w[B] = 0u;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        uint32_t par = 0, dg[8];
        const int base = b * 8 * B;
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            dg[i] = field(w, base + i * B, B);
            par ^= dg[i];
        }
        const uint32_t f7 = field(w, base + 7 * B, B);
        dg[7] = (f7 & ~1u) | (par & 1u);
        const float* t = lev + ((f7 & 1u) ? (1 << B) : 0);
#pragma unroll
        for (int i = 0; i < 8; ++i) Lb[(kk0 + b * 8 + i) * kVT + v] = live ? __fmul_rn(cf, __ldg(t + dg[i])) : 0.0f;
    }
}

// ME8Q persistent scan: the batched kernel's structure with one rate per
// 64-dim chunk (a run never splits a chunk). With the coef of each segment
// folded into its decoded levels, sum_s coef_s S_s is one contraction q . L',
// and the estimator d2 + sum_s (h2_s - 2 coef_s S_s) (src/index/
// me8q_search.cpp:74-95) becomes d2 + hsum - 2 q . L'.
__global__ void __launch_bounds__(kBT) me8q_scan_kernel(
    Me8qView mv, const float* __restrict__ rq, const uint4* __restrict__ items, const uint32_t* __restrict__ n_items,
    uint32_t* __restrict__ head, const uint32_t* __restrict__ pair_q, const float* __restrict__ pair_d2,
    const uint32_t* __restrict__ k_arr, int k_uniform, int k_max, float* __restrict__ part_d,
    uint32_t* __restrict__ part_id, unsigned long long* __restrict__ cand_count) {
    extern __shared__ __align__(16) float bsm[];
    const DevIndex& ix = mv.base;
    float* Qs = bsm;                 // 2 * kKC * kQT
    float* Ls = Qs + 2 * kKC * kQT;  // 2 * kKC * kVT
    float* tk_d = Ls + 2 * kKC * kVT;
    uint32_t* tk_i = reinterpret_cast<uint32_t*>(tk_d + kQT * k_max);
    __shared__ uint4 s_item;
    __shared__ uint32_t s_q[kQT];
    __shared__ float s_d2[kQT];
    __shared__ int s_k[kQT];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int pd = ix.pd;
    const int nK = mv.nchunks;
    const int tq = tid >> 4, tv = tid & 15;
    const uint32_t NI = *n_items;
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
        if (tid < kQT) {
            const bool ok = tid < m;
            const uint32_t qq = ok ? pair_q[pbase + tid] : 0u;
            s_q[tid] = qq;
            s_d2[tid] = ok ? pair_d2[pbase + tid] : 0.0f;
            s_k[tid] = ok ? (k_arr ? static_cast<int>(k_arr[qq]) : k_uniform) : 0;
        }
        for (int e = tid; e < kQT * k_max; e += kBT) {
            tk_d[e] = inf_f();
            tk_i[e] = 0xFFFFFFFFu;
        }
        __syncthreads();
        const uint32_t len = ix.list_len[L];
        const uint32_t tile0 = ix.tile_begin[L];
        if (tid == 0) {
            atomicAdd(cand_count, static_cast<unsigned long long>(len) * m);
            atomicAdd(cand_count + 1, static_cast<unsigned long long>(len));
            if (item.w == 0) atomicAdd(cand_count + 2, static_cast<unsigned long long>(len));
        }
        for (uint32_t v0 = 0; v0 < len; v0 += kVT) {
            float acc[4][8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;
            for (int kc = 0; kc < nK; ++kc) {
                float* Qb = Qs + (kc & 1) * kKC * kQT;
                float* Lb = Ls + (kc & 1) * kKC * kVT;
                {
                    const int q = tid & 63, part = tid >> 6;
                    const float* src = rq + static_cast<size_t>(s_q[q]) * pd + kc * kKC + part * 16;
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const float4 val = q < m ? *reinterpret_cast<const float4*>(src + 4 * r)
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
                        const int kk = part * 16 + 4 * r;
                        Qb[(kk + 0) * kQT + q] = val.x;
                        Qb[(kk + 1) * kQT + q] = val.y;
                        Qb[(kk + 2) * kQT + q] = val.z;
                        Qb[(kk + 3) * kQT + q] = val.w;
                    }
                }
                {
                    const Me8qChunk ch = mv.chunks[kc];
                    const int v = tid & 127, h = tid >> 7;
                    const uint32_t vi = v0 + v;
                    const bool live = vi < len;
                    const uint32_t gt = tile0 + (vi >> 5);
                    const int vl = static_cast<int>(vi & 31);
                    const size_t slot = static_cast<size_t>(gt) * 32 + vl;
                    const float cf = live && ch.coded >= 0
                                         ? __ldg(mv.coef + static_cast<size_t>(ch.coded) * mv.nslots + slot)
                                         : 0.0f;
                    const int w0 = ch.word0 + h * ch.bits;  // 4 blocks = bits words
                    const float* lev = mv.levels + ch.lev;
                    switch (ch.bits) {
#define E8QC_DEC(B) \
    case B: me8q_decode_half<B>(ix, gt, vl, live, w0, lev, cf, Lb, h * 32, v); break;
                        E8QC_DEC(1) E8QC_DEC(2) E8QC_DEC(3) E8QC_DEC(4) E8QC_DEC(5) E8QC_DEC(6) E8QC_DEC(7)
                        E8QC_DEC(8) E8QC_DEC(9) E8QC_DEC(10) E8QC_DEC(11) E8QC_DEC(12) E8QC_DEC(13)
#undef E8QC_DEC
                        default:  // a dropped run inside the coded prefix contributes nothing
                            for (int i = 0; i < 32; ++i) Lb[(h * 32 + i) * kVT + v] = 0.0f;
                            break;
                    }
                }
                __syncthreads();
#pragma unroll 4
                for (int kk = 0; kk < kKC; ++kk) {
                    const float4 a = *reinterpret_cast<const float4*>(Qb + kk * kQT + tq * 4);
                    const float4 b0 = *reinterpret_cast<const float4*>(Lb + kk * kVT + tv * 4);
                    const float4 b1 = *reinterpret_cast<const float4*>(Lb + kk * kVT + 64 + tv * 4);
                    const float av[4] = {a.x, a.y, a.z, a.w};
                    const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[i][j] = __fmaf_rn(av[i], bv[j], acc[i][j]);
                }
            }
            __syncthreads();
            float* D = Ls;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int vv = j < 4 ? tv * 4 + j : 64 + tv * 4 + (j - 4);
                const uint32_t vi = v0 + vv;
                const bool live = vi < len;
                const size_t slot = static_cast<size_t>(tile0 + (vi >> 5)) * 32 + (vi & 31);
                const float hs = live ? __ldg(mv.hsum + slot) : 0.0f;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int q = tq * 4 + i;
                    D[q * kVT + vv] = live ? __fmaf_rn(-2.0f, acc[i][j], __fadd_rn(s_d2[q], hs)) : inf_f();
                }
            }
            __syncthreads();
            for (int q = warp; q < m; q += kBT / 32) {
                const int kq = s_k[q];
                WarpTopK top;
                top.init(kq);
#pragma unroll
                for (int s2 = 0; s2 < 4; ++s2) {
                    const int j = s2 * 32 + lane;
                    if (j < kq) {
                        top.d[s2] = tk_d[q * k_max + j];
                        top.id[s2] = tk_i[q * k_max + j];
                    }
                }
                top.refresh_threshold();
                for (int c = 0; c < kVT; c += 32) {
                    const uint32_t vi = v0 + c + lane;
                    const bool live = vi < len;
                    const float dist = D[q * kVT + c + lane];
                    const size_t slot = static_cast<size_t>(tile0 + (vi >> 5)) * 32 + (vi & 31);
                    top.offer(dist, live, [&] { return __ldg(ix.ids + slot); });
                }
                top.store(tk_d + q * k_max, tk_i + q * k_max, kq);
            }
            __syncthreads();
        }
        for (int e = tid; e < m * k_max; e += kBT) {
            const int q = e / k_max, j = e - q * k_max;
            const size_t o = static_cast<size_t>(pbase + q) * k_max + j;
            part_d[o] = tk_d[e];
            part_id[o] = tk_i[e];
        }
    }
}

// Per-query merge of its nprobe partial lists into the final top-k row.
__global__ void merge_kernel(const float* __restrict__ part_d, const uint32_t* __restrict__ part_id,
                             const uint32_t* __restrict__ pos_of, int nq, const uint32_t* __restrict__ np_arr,
                             int np_uniform, int np_max, const uint32_t* __restrict__ k_arr, int k_uniform,
                             int k_max, int out_stride, uint32_t* __restrict__ out_ids, float* __restrict__ out_d) {
    const int lane = threadIdx.x & 31;
    const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (q >= nq) return;
    const int np = np_arr ? static_cast<int>(np_arr[q]) : np_uniform;
    const int kq = k_arr ? static_cast<int>(k_arr[q]) : k_uniform;
    WarpTopK top;
    top.init(kq);
    const int total = np * kq;
    for (int e0 = 0; e0 < total; e0 += 32 * 4) {
        float dd[4];
        uint32_t ii[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = e0 + r * 32 + lane;
            dd[r] = inf_f();
            ii[r] = 0xFFFFFFFFu;
            if (e < total) {
                const int p = e / kq, j = e - p * kq;
                const size_t o = static_cast<size_t>(pos_of[static_cast<size_t>(q) * np_max + p]) * k_max + j;
                dd[r] = part_d[o];
                ii[r] = part_id[o];
            }
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) top.offer_pair(dd[r], ii[r], ii[r] != 0xFFFFFFFFu);
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

}  // namespace

size_t batched_scan_smem(const DevIndex& ix, int k_max);

namespace {
template <int BITS>
void launch_batched_scan(const DevIndex& ix, const float* rq, Workspace& ws, uint32_t* nitems,
                         const uint32_t* k_arr, int k_max, size_t smem, int dev, cudaStream_t s) {
    static size_t configured[64] = {};
    if (configured[dev & 63] < smem) {
        E8QC_CUDA(cudaFuncSetAttribute(batched_scan_kernel<BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        configured[dev & 63] = smem;
    }
    int sms = 148, per_sm = 1;
    E8QC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    E8QC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_scan_kernel<BITS>, kBT, smem));
    per_sm = std::max(1, per_sm);
    batched_scan_kernel<BITS><<<sms * per_sm, kBT, smem, s>>>(
        ix, rq, ws.b_items.as<uint4>(), nitems, nitems + 1, ws.b_pair_q.as<uint32_t>(), ws.b_pair_d2.as<float>(),
        k_arr, k_max, k_max, ws.b_part_d.as<float>(), ws.b_part_id.as<uint32_t>(),
        reinterpret_cast<unsigned long long*>(nitems + 2));
}
}  // namespace

size_t batched_scan_smem(const DevIndex& ix, int k_max) {
    return (static_cast<size_t>(2) * kKC * kQT + 2 * kKC * kVT + 2 * (1 << ix.bits) + 2 * kQT * k_max) * 4;
}

int group_pairs(const DevIndex& ix, Workspace& ws, size_t nq, const uint32_t* np_arr, int np_max, size_t pslots,
                size_t item_cap, int qt, int align, cudaStream_t s);

int batched_prepare(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* np_arr,
                    size_t nprobe, size_t part_width, int qt, int align, cudaStream_t s) {
    const int nlist = ix.nlist;
    const int np_max = static_cast<int>(nprobe);
    const size_t npairs = nq * static_cast<size_t>(np_max);
    // pair slots: aligned list starts leave up to align-1 unused slots per list
    const size_t pslots = npairs + static_cast<size_t>(align - 1) * nlist;
    // upper bound of items: pairs/qt + one partial item per list
    const size_t item_cap = npairs / qt + static_cast<size_t>(nlist) + 1;
    ws.b_keys.ensure(nq * static_cast<size_t>(nlist) * 8);
    ws.b_qn2.ensure(nq * 4);
    ws.b_probes.ensure(npairs * 4);
    ws.b_pd2.ensure(npairs * 4);
    ws.b_pos.ensure(npairs * 4);
    ws.b_pair_q.ensure(pslots * 4);
    ws.b_pair_d2.ensure(pslots * 4);
    ws.b_cnt.ensure(static_cast<size_t>(nlist) * 4);
    ws.b_off.ensure(static_cast<size_t>(nlist) * 4);
    ws.b_fill.ensure(static_cast<size_t>(nlist) * 4);
    ws.b_items.ensure(item_cap * 16);
    ws.b_nitems.ensure(48);
    ws.b_part_d.ensure(npairs * part_width * 4);
    ws.b_part_id.ensure(npairs * part_width * 4);
    int launches = 0;
    qn2_kernel<<<static_cast<unsigned>(nq), 256, 0, s>>>(rq, ix.pd, ws.b_qn2.as<float>());
    ++launches;
    E8QC_CUDA(cudaMemsetAsync(ws.b_cnt.p, 0, static_cast<size_t>(nlist) * 4, s));
    E8QC_CUDA(cudaMemsetAsync(ws.b_nitems.p, 0, 48, s));  // [0] n_items, [1] head, [2..7] pair / vector / list-vector counts
    if (ws.route_tc && route_tc_applies(ix, nq)) {
        launches += route_tc_keys(ix, ws, rq, nq, s);
    } else {
        if (ix.pd % kRouteBK != 0)
            fail(E8QC_EINVAL, "batched route needs the padded dimension to be a multiple of 16");
        dim3 g((nlist + kRouteBC - 1) / kRouteBC, static_cast<unsigned>((nq + kRouteBQ - 1) / kRouteBQ));
        route_gemm_kernel<<<g, 128, 0, s>>>(rq, static_cast<int>(nq), ix.cen, ix.cn2, nlist, ix.pd,
                                            ws.b_qn2.as<float>(), ws.b_keys.as<uint64_t>());
        ++launches;
    }
    const size_t sel_smem = static_cast<size_t>(nlist) * 8;  // d2 words + interval lower bounds
    if (sel_smem > 200 * 1024) fail(E8QC_EINVAL, "batched route supports at most 25600 lists");
    {
        // raised once per device (also keeps the call out of captured sequences)
        int dev = 0;
        E8QC_CUDA(cudaGetDevice(&dev));
        static size_t configured[64] = {};
        if (sel_smem > 48 * 1024 && configured[dev & 63] < sel_smem) {
            E8QC_CUDA(cudaFuncSetAttribute(select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(sel_smem)));
            configured[dev & 63] = sel_smem;
        }
    }
    select_kernel<<<static_cast<unsigned>(nq), 256, sel_smem, s>>>(
        ws.b_keys.as<uint64_t>(), ws.r_ub.as<uint32_t>(), nlist, np_arr, np_max, np_max, rq, ix.cen, ix.pd,
        ws.b_qn2.as<float>(), ix.cn2, ws.b_probes.as<uint32_t>(), ws.b_pd2.as<float>(), ws.b_cnt.as<uint32_t>());
    ++launches;
    return launches + group_pairs(ix, ws, nq, np_arr, np_max, pslots, item_cap, qt, align, s);
}

// Work items and the (query, list) pair arrays from the probes and per-list
// pair counts of a routed batch.
int group_pairs(const DevIndex& ix, Workspace& ws, size_t nq, const uint32_t* np_arr, int np_max, size_t pslots,
                size_t item_cap, int qt, int align, cudaStream_t s) {
    const int nlist = ix.nlist;
    const size_t npairs = nq * static_cast<size_t>(np_max);
    int launches = 0;
    uint32_t* nitems = ws.b_nitems.as<uint32_t>();
    items_kernel<<<1, 1024, 0, s>>>(ws.b_cnt.as<uint32_t>(), ix.list_order + (ws.sched ? nlist : 0), nlist,
                                    ws.b_off.as<uint32_t>(),
                                    ws.b_fill.as<uint32_t>(), ws.b_items.as<uint4>(), nitems,
                                    static_cast<int>(item_cap), static_cast<uint32_t>(qt),
                                    static_cast<uint32_t>(align));
    ++launches;
    // unused slots keep the query id UINT32_MAX
    if (align > 1) E8QC_CUDA(cudaMemsetAsync(ws.b_pair_q.p, 0xFF, pslots * 4, s));
    scatter_kernel<<<static_cast<unsigned>((npairs + 255) / 256), 256, 0, s>>>(
        ws.b_probes.as<uint32_t>(), ws.b_pd2.as<float>(), static_cast<int>(nq), np_arr, np_max, np_max,
        ws.b_off.as<uint32_t>(), ws.b_fill.as<uint32_t>(), ws.b_pair_q.as<uint32_t>(), ws.b_pair_d2.as<float>(),
        ws.b_pos.as<uint32_t>());
    ++launches;
    E8QC_CUDA(cudaGetLastError());
    return launches;
}

int batched_search(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                   const uint32_t* np_arr, size_t k, size_t nprobe, size_t out_stride, uint32_t* out_ids,
                   float* out_d, size_t max_tiles, cudaStream_t s) {
    (void)max_tiles;
    if (nq == 0) return 0;
    const int k_max = static_cast<int>(k);
    const int np_max = static_cast<int>(nprobe);
    int launches = batched_prepare(ix, ws, rq, nq, np_arr, nprobe, k, kQT, 1, s);
    uint32_t* nitems = ws.b_nitems.as<uint32_t>();
    const size_t smem = batched_scan_smem(ix, k_max);
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    ws.mark_scan(false, s);
    switch (ix.bits) {
#define E8QC_CASE(b) \
    case b: launch_batched_scan<b>(ix, rq, ws, nitems, k_arr, k_max, smem, dev, s); break;
        E8QC_CASE(1) E8QC_CASE(2) E8QC_CASE(3) E8QC_CASE(4) E8QC_CASE(5) E8QC_CASE(6)
        E8QC_CASE(7) E8QC_CASE(8) E8QC_CASE(9) E8QC_CASE(10) E8QC_CASE(11) E8QC_CASE(12)
        E8QC_CASE(13)
#undef E8QC_CASE
        default: fail(E8QC_EINVAL, "bits out of range");
    }
    ws.mark_scan(true, s);
    ++launches;
    merge_kernel<<<static_cast<unsigned>((nq + 3) / 4), 128, 0, s>>>(
        ws.b_part_d.as<float>(), ws.b_part_id.as<uint32_t>(), ws.b_pos.as<uint32_t>(), static_cast<int>(nq), np_arr,
        np_max, np_max, k_arr, k_max, k_max, static_cast<int>(out_stride), out_ids, out_d);
    ++launches;
    E8QC_CUDA(cudaGetLastError());
    return launches;
}

int me8q_grouped_search(const Me8qView& v, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                        const uint32_t* np_arr, size_t k, size_t nprobe, size_t out_stride, uint32_t* out_ids,
                        float* out_d, cudaStream_t s) {
    if (nq == 0) return 0;
    const int k_max = static_cast<int>(k);
    const int np_max = static_cast<int>(nprobe);
    int launches = batched_prepare(v.base, ws, rq, nq, np_arr, nprobe, k, kQT, 1, s);
    int dev = 0;
    E8QC_CUDA(cudaGetDevice(&dev));
    const size_t smem = (static_cast<size_t>(2) * kKC * kQT + 2 * kKC * kVT + 2 * kQT * k_max) * 4;
    static size_t configured[64] = {};
    if (configured[dev & 63] < smem) {
        E8QC_CUDA(cudaFuncSetAttribute(me8q_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        configured[dev & 63] = smem;
    }
    int sms = 148, per_sm = 1;
    E8QC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    E8QC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, me8q_scan_kernel, kBT, smem));
    per_sm = std::max(1, per_sm);
    uint32_t* nitems = ws.b_nitems.as<uint32_t>();
    ws.mark_scan(false, s);
    me8q_scan_kernel<<<sms * per_sm, kBT, smem, s>>>(
        v, rq, ws.b_items.as<uint4>(), nitems, nitems + 1, ws.b_pair_q.as<uint32_t>(), ws.b_pair_d2.as<float>(), k_arr,
        k_max, k_max, ws.b_part_d.as<float>(), ws.b_part_id.as<uint32_t>(),
        reinterpret_cast<unsigned long long*>(nitems + 2));
    E8QC_CUDA(cudaGetLastError());
    ws.mark_scan(true, s);
    ++launches;
    merge_kernel<<<static_cast<unsigned>((nq + 3) / 4), 128, 0, s>>>(
        ws.b_part_d.as<float>(), ws.b_part_id.as<uint32_t>(), ws.b_pos.as<uint32_t>(), static_cast<int>(nq), np_arr,
        np_max, np_max, k_arr, k_max, k_max, static_cast<int>(out_stride), out_ids, out_d);
    E8QC_CUDA(cudaGetLastError());
    return launches + 1;
}

}  // namespace e8qc
