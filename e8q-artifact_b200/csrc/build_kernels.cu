// Build-path kernels: the fp64 mean, centroid rotation, and the fused
// rotate -> residual -> E8 encode -> fit -> pack kernel, plus the standalone
// encoder and the code export.
//
// This translation unit is compiled with --fmad=false: the encoder's integer
// choices depend on fp64 costs, and the reference computes them without
// contraction. The accumulations the reference's GCC build does fuse
// (residual norm, the g1/h3 fit sums) are written as __fma_rn.
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "device_common.cuh"
#include "internal.h"

namespace e8qc {

namespace {

// ---------------------------------------------------------------------------
// Encoder primitives (src/quantization/e8q_codec.cpp).

// First index with lev[i] >= v (std::lower_bound), through the bounded-bin
// index when usable: e8q_codec.cpp:190-231, :354-385.
__device__ __forceinline__ int insert_pos(const DevLevelTable& t, double v) {
    const double* lev = t.lev;
    const int n = t.n;
    if (t.usable) {
        if (v <= t.bin_lo_v) return 0;
        if (v > lev[n - 1]) return n;
        long bin = static_cast<long>((v - t.bin_lo_v) * t.bin_scale);
        if (bin >= t.nbins) bin = t.nbins - 1;
        int pos = static_cast<int>(t.bin_lo[bin]);
        pos += (lev[pos] < v) ? 1 : 0;
        pos += (lev[pos] < v) ? 1 : 0;
        return pos;
    }
    int pos = 0, step = 1;
    while (step * 2 <= n) step *= 2;
    for (; step != 0; step >>= 1) {
        const int next = pos + step;
        pos += (next <= n && lev[next - 1] < v) ? step : 0;
    }
    return pos;
}

// Nearest level of each class r (= 2*parity + branch) of the merged table:
// e8q_codec.cpp:392-414.
__device__ __forceinline__ void nearest_merged(double v, const DevLevelTable& t, uint16_t dig[4],
                                               double cost[4]) {
    const int p = insert_pos(t, v);
    const int p4 = p & 3;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i_b = p - 1 - ((p4 + 3 - r) & 3);
        const int i_a = p + ((r + 4 - p4) & 3);
        const uint16_t d_b = t.dig[i_b], d_a = t.dig[i_a];
        const double dv_b = v - t.lev[i_b];
        const double dv_a = t.lev[i_a] - v;
        const double c_b = dv_b * dv_b, c_a = dv_a * dv_a;
        const bool take_b = (c_b < c_a) | ((c_b == c_a) & (d_b < d_a));
        dig[r] = take_b ? d_b : d_a;
        cost[r] = take_b ? c_b : c_a;
    }
}

// Nearest level in one (branch, parity) table: e8q_codec.cpp:233-256.
__device__ __forceinline__ void nearest_in_table(double v, const DevLevelTable& t, uint16_t* digit,
                                                 double* cost) {
    const int n = t.n;
    const int pos = insert_pos(t, v);
    int best = pos < n ? pos : n - 1;
    if (pos > 0) {
        const double dc = fabs(v - t.lev[pos - 1]);
        const double db = fabs(v - t.lev[best]);
        const uint16_t dig_c = t.dig[pos - 1], dig_b = t.dig[best];
        const bool take_below = (dc < db) | ((dc == db) & (dig_c < dig_b));
        best = take_below ? pos - 1 : best;
    }
    *digit = t.dig[best];
    const double dv = v - t.lev[best];
    *cost = dv * dv;
}

// Per-coordinate parity choice + single-flip parity repair:
// e8q_codec.cpp:549-599. Returns the block cost.
__device__ __forceinline__ double assemble(const uint16_t de[8], const double ce[8],
                                           const uint16_t dodd[8], const double co[8],
                                           uint16_t out[8]) {
    double cost = 0.0;
    int parity = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const bool use_odd = co[i] < ce[i];
        out[i] = use_odd ? dodd[i] : de[i];
        cost += use_odd ? co[i] : ce[i];
        parity ^= use_odd ? 1 : 0;
    }
    if (parity != 0) {
        int sel = 0;
        double best_extra = DBL_MAX;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const bool was_odd = out[i] == dodd[i];
            const double extra = was_odd ? ce[i] - co[i] : co[i] - ce[i];
            if (extra < best_extra) {
                best_extra = extra;
                sel = i;
            }
        }
        const bool was_odd = out[sel] == dodd[sel];
        out[sel] = was_odd ? de[sel] : dodd[sel];
        cost += (best_extra < 0.0) ? 0.0 : best_extra;
    }
    return cost;
}

// One 8-d block of scaled values -> digits + branch (EncodeVectorAtScaleInto's
// per-block body, e8q_codec.cpp:685-725): both branches from one merged
// search per coordinate when the merged table alternates, else from the four
// parity tables; branch 1 only when strictly cheaper.
__device__ int encode_block(const double v[8], const DevEncTables& et, uint16_t out[8]) {
    uint16_t d0[8], d1[8];
    double c0, c1;
    if (et.alternating) {
        uint16_t de0[8], do0[8], de1[8], do1[8];
        double ce0[8], co0[8], ce1[8], co1[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint16_t dg[4];
            double cs[4];
            nearest_merged(v[i], et.merged, dg, cs);
            de0[i] = dg[0]; ce0[i] = cs[0];
            de1[i] = dg[1]; ce1[i] = cs[1];
            do0[i] = dg[2]; co0[i] = cs[2];
            do1[i] = dg[3]; co1[i] = cs[3];
        }
        c0 = assemble(de0, ce0, do0, co0, d0);
        c1 = assemble(de1, ce1, do1, co1, d1);
    } else {
        uint16_t de[8], dodd[8];
        double ce[8], co[8];
        for (int i = 0; i < 8; ++i) {
            nearest_in_table(v[i], et.parity[0], &de[i], &ce[i]);
            nearest_in_table(v[i], et.parity[1], &dodd[i], &co[i]);
        }
        c0 = assemble(de, ce, dodd, co, d0);
        for (int i = 0; i < 8; ++i) {
            nearest_in_table(v[i], et.parity[2], &de[i], &ce[i]);
            nearest_in_table(v[i], et.parity[3], &dodd[i], &co[i]);
        }
        c1 = assemble(de, ce, dodd, co, d1);
    }
    const bool take1 = c1 < c0;
#pragma unroll
    for (int i = 0; i < 8; ++i) out[i] = take1 ? d1[i] : d0[i];
    return take1 ? 1 : 0;
}

// ---------------------------------------------------------------------------
// fp64 mean of the build rows in file order (src/index/e8q_build.cpp:190-204):
// one thread per dimension summing rows 0..n-1 sequentially, so the sum has
// the reference's exact rounding sequence.
__global__ void mean_kernel(const float* __restrict__ x, size_t n, int dim, float* __restrict__ mu) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= dim) return;
    double s = 0.0;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = __ldg(x + (i + j) * dim + d);
#pragma unroll
        for (int j = 0; j < 8; ++j) s += static_cast<double>(v[j]);
    }
    for (; i < n; ++i) s += static_cast<double>(__ldg(x + i * dim + d));
    mu[d] = static_cast<float>(s / static_cast<double>(n));
}

// Rotated, centred centroids and their fp64 norms (e8q_build.cpp:249-272).
__global__ void centroids_kernel(const uint8_t* __restrict__ signs, int dim, int pd, int td, float fac,
                                 const float* __restrict__ raw, const float* __restrict__ mean_rot,
                                 float* __restrict__ out, float* __restrict__ cn2) {
    extern __shared__ float sx[];
    const size_t c = blockIdx.x;
    for (int i = threadIdx.x; i < pd; i += blockDim.x) sx[i] = i < dim ? raw[c * dim + i] : 0.0f;
    __syncthreads();
    rotate_rows_smem(sx, 1, pd, pd, td, fac, signs);
    for (int i = threadIdx.x; i < pd; i += blockDim.x) {
        sx[i] = __fsub_rn(sx[i], mean_rot[i]);
        out[c * pd + i] = sx[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < pd; ++i) s = __fma_rn(static_cast<double>(sx[i]), static_cast<double>(sx[i]), s);
        cn2[c] = static_cast<float>(s);
    }
}

// Fused build of RB slots of one tile: rotate the raw rows, centre, residual
// against the list's rotated centroid, unit = float(residual / ||residual||),
// encode every block, fit g1 = rn/<u,vE> and h3 = rn^2 + 2*g1*<c,vE>, and pack
// the device code layout. Follows src/index/e8q_build.cpp:306-418.
constexpr int kBuildThreads = 256;

// Shared-memory carve of build_encode_kernel (16-byte aligned sections).
struct BuildSmem {
    size_t x, c, rn, dig, br, words, total;
    __host__ __device__ static size_t up(size_t v) { return (v + 15) & ~size_t(15); }
    __host__ __device__ BuildSmem(int rb, int pd, int B, int nch) {
        x = 0;
        c = up(x + static_cast<size_t>(rb) * (pd + 1) * 4);
        rn = up(c + static_cast<size_t>(pd) * 4);
        dig = up(rn + static_cast<size_t>(rb) * 8);
        br = up(dig + static_cast<size_t>(rb) * B * 8 * 2);
        words = up(br + static_cast<size_t>(rb) * B);
        total = up(words + static_cast<size_t>(rb) * nch * 16);
    }
};

__global__ void __launch_bounds__(kBuildThreads) build_encode_kernel(
    DevIndex ix, DevEncTables et, BuildEncodeArgs a, int rb, int td, float fac,
    uint4* __restrict__ codes, float* __restrict__ g1o, float* __restrict__ h3o) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int pd = ix.pd, B = ix.B, bits = ix.bits, nch = ix.nch;
    const int ld = pd + 1;
    const BuildSmem L(rb, pd, B, nch);
    float* X = reinterpret_cast<float*>(smraw + L.x);          // rb * ld
    float* C = reinterpret_cast<float*>(smraw + L.c);          // pd
    double* rn2s = reinterpret_cast<double*>(smraw + L.rn);    // rb
    uint16_t* dig = reinterpret_cast<uint16_t*>(smraw + L.dig); // rb * B * 8
    uint8_t* brs = smraw + L.br;                                // rb * B
    uint32_t* words = reinterpret_cast<uint32_t*>(smraw + L.words);  // rb * nch * 4
    __shared__ uint32_t rows[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per_tile = 32 / rb;
    const int tile = blockIdx.x / per_tile;
    const int lane0 = (blockIdx.x % per_tile) * rb;
    const uint32_t list = a.list_of_tile[tile];
    if (tid < rb) rows[tid] = a.row_of[static_cast<size_t>(tile) * 32 + lane0 + tid];
    __syncthreads();
    for (int e = tid; e < rb * pd; e += nt) {
        const int r = e / pd, i = e - r * pd;
        const uint32_t row = rows[r];
        X[r * ld + i] = (row != 0xFFFFFFFFu && i < ix.dim) ? a.base[static_cast<size_t>(row) * ix.dim + i] : 0.0f;
    }
    for (int i = tid; i < pd; i += nt) C[i] = ix.cen[static_cast<size_t>(list) * pd + i];
    for (int e = tid; e < rb * nch * 4; e += nt) words[e] = 0u;
    __syncthreads();
    rotate_rows_smem(X, rb, ld, pd, td, fac, ix.signs);
    for (int e = tid; e < rb * pd; e += nt) {
        const int r = e / pd, i = e - r * pd;
        X[r * ld + i] = __fsub_rn(X[r * ld + i], ix.mean_rot[i]);
    }
    __syncthreads();
    // residual norm, sequential over the dimension (fused, as the reference build)
    if (tid < rb) {
        double s = 0.0;
        for (int i = 0; i < pd; ++i) {
            const double rv = static_cast<double>(X[tid * ld + i]) - static_cast<double>(C[i]);
            s = __fma_rn(rv, rv, s);
        }
        rn2s[tid] = s;
    }
    __syncthreads();
    for (int e = tid; e < rb * pd; e += nt) {
        const int r = e / pd, i = e - r * pd;
        const double rn = sqrt(rn2s[r]);
        const double inv = 1.0 / rn;
        X[r * ld + i] = static_cast<float>((static_cast<double>(X[r * ld + i]) - static_cast<double>(C[i])) * inv);
    }
    __syncthreads();
    // encode: one thread per (row, block)
    for (int e = tid; e < rb * B; e += nt) {
        const int r = e / B, blk = e - r * B;
        const bool live = rows[r] != 0xFFFFFFFFu && !(sqrt(rn2s[r]) < 1e-20);
        uint16_t out[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int br = 0;
        if (live) {
            double v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = static_cast<double>(X[r * ld + blk * 8 + i]) * a.srd;
            br = encode_block(v, et, out);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) dig[(r * B + blk) * 8 + i] = out[i];
        brs[r * B + blk] = static_cast<uint8_t>(br);
        // pack: digit i at bit blk*8*bits + i*bits; digit 7's LSB slot = branch
        const int base = blk * 8 * bits;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint32_t f = out[i] & ((1u << bits) - 1u);
            if (i == 7) f = (f & ~1u) | static_cast<uint32_t>(br);
            const int off = base + i * bits;
            const int wi = off >> 5, sh = off & 31;
            if (f) {
                atomicOr(&words[r * nch * 4 + wi], f << sh);
                if (sh + bits > 32) atomicOr(&words[r * nch * 4 + wi + 1], f >> (32 - sh));
            }
        }
    }
    __syncthreads();
    // fits, sequential per row (fused accumulations, as the reference build)
    if (tid < rb) {
        const int r = tid;
        const size_t slot = static_cast<size_t>(tile) * 32 + lane0 + r;
        float g1f = 0.0f, h3f = 0.0f, obf = 0.0f, owf = 0.0f, opf = 0.0f;
        const double rn2 = rn2s[r];
        const double rn = sqrt(rn2);
        if (rows[r] != 0xFFFFFFFFu && !(rn < 1e-20)) {
            double dot_ue = 0.0, n2_e = 0.0, dot_ce = 0.0;
            // scan-basis projections (e8q_build.cpp:338-377): w is the class
            // mean of each digit's top bit, none for dim 7 at b = 1
            double dot_ew = 0.0, dot_uw = 0.0, n2_w = 0.0, dot_cw = 0.0;
            for (int blk = 0; blk < B; ++blk) {
                const double* lv = et.levels[brs[r * B + blk]];
                for (int kk = 0; kk < 8; ++kk) {
                    const int idx = blk * 8 + kk;
                    const int digit = dig[(r * B + blk) * 8 + kk];
                    const double ve = lv[digit] * a.inv_level_scale;
                    const double wc = (bits == 1 && kk == 7) ? 0.0 : a.w_cls[digit >> (bits - 1)];
                    const double u = static_cast<double>(X[r * ld + idx]), cc = static_cast<double>(C[idx]);
                    dot_ue = __fma_rn(u, ve, dot_ue);
                    dot_ce = __fma_rn(cc, ve, dot_ce);
                    n2_e = __fma_rn(ve, ve, n2_e);
                    dot_ew = __fma_rn(ve, wc, dot_ew);
                    dot_uw = __fma_rn(u, wc, dot_uw);
                    n2_w = __fma_rn(wc, wc, n2_w);
                    dot_cw = __fma_rn(cc, wc, dot_cw);
                }
            }
            if (n2_e > 1e-30 && dot_ue > 1e-12) {
                const double g1 = rn / dot_ue;
                const double h3 = __fma_rn(2.0 * g1, dot_ce, rn2);
                g1f = static_cast<float>(g1);
                h3f = static_cast<float>(h3);
            }
            // orthogonal-projection bank inputs (e8q_build.cpp:414-445), with
            // the reference build's fused multiply-adds spelled out
            const double g1v = static_cast<double>(g1f);
            const double sqrt_dm1 = sqrt(static_cast<double>(ix.dim > 1 ? ix.dim - 1 : 1));
            const double n2_w_safe = n2_w < 1e-30 ? 1e-30 : n2_w;
            const double uw_eps = 1e-12 * sqrt(n2_w_safe);
            double w_use, perp_use;
            if (fabs(dot_uw) > uw_eps) {
                const double wx = 2.0 * rn / dot_uw;
                const double a1 = 4.0 * g1v * g1v, b1 = wx * wx, c1 = 4.0 * g1v * wx;
                const double rx2 = __fma_rn(-c1, dot_ew, __fma_rn(a1, n2_e, b1 * n2_w));
                w_use = wx;
                perp_use = sqrt(0.0 < rx2 ? rx2 : 0.0) / sqrt_dm1;
            } else {
                const double gamma = dot_ew / n2_w_safe;
                const double t = __fma_rn(-(gamma * gamma), n2_w, n2_e);
                const double vp2 = t < 0.0 ? 0.0 : t;
                w_use = 2.0 * g1v * gamma;
                perp_use = 2.0 * g1v * sqrt(vp2) / sqrt_dm1;
            }
            owf = static_cast<float>(w_use);
            obf = static_cast<float>(__fma_rn(w_use, dot_cw, rn2));
            opf = static_cast<float>(perp_use);
        }
        g1o[slot] = g1f;
        h3o[slot] = h3f;
        if (a.ortho) {
            a.ortho[slot * 3 + 0] = obf;
            a.ortho[slot * 3 + 1] = owf;
            a.ortho[slot * 3 + 2] = opf;
        }
    }
    // write the tile's chunks: chunk c of lane l at [tile][c][l]
    for (int e = tid; e < rb * nch; e += nt) {
        const int r = e / nch, c = e - r * nch;
        const uint32_t* wp = words + (r * nch + c) * 4;
        codes[(static_cast<size_t>(tile) * nch + c) * 32 + lane0 + r] = make_uint4(wp[0], wp[1], wp[2], wp[3]);
    }
}

// Standalone encoder: one thread per (vector, block).
__global__ void encode_kernel(DevEncTables et, const float* __restrict__ unit, size_t n, int pd,
                              double srd, uint16_t* __restrict__ digits, uint8_t* __restrict__ branch) {
    const int B = pd / 8;
    const size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n * static_cast<size_t>(B)) return;
    const size_t r = e / B;
    const int blk = static_cast<int>(e - r * B);
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = static_cast<double>(unit[r * pd + blk * 8 + i]) * srd;
    uint16_t out[8];
    const int br = encode_block(v, et, out);
#pragma unroll
    for (int i = 0; i < 8; ++i) digits[e * 8 + i] = out[i];
    branch[e] = static_cast<uint8_t>(br);
}

// ME8Q segment encoder (SegmentCodec::EncodeInto, src/quantization/
// me8q_codec.cpp:69-97): one thread per (row, block) of one coded run. The
// run's rotated residual rr and its fp64 norm^2 give unit = float(rr * (1 /
// sqrt(norm^2))); the block is then encoded like an E8Q block of a len-dim
// vector (scale * sqrt(len)). A zero-norm run stays the all-zero codeword.
__global__ void me8q_encode_kernel(DevEncTables et, const float* __restrict__ rr, int pd,
                                   const double* __restrict__ norm2, int ncoded, int run, int off, int len,
                                   size_t n, double srd, uint16_t* __restrict__ digits,
                                   uint8_t* __restrict__ branch) {
    const int nb = len / 8;
    const size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= n * static_cast<size_t>(nb)) return;
    const size_t r = e / nb;
    const int blk = static_cast<int>(e - r * nb);
    uint16_t* dg = digits + r * pd + off + blk * 8;
    const double n2 = norm2[r * ncoded + run];
    if (!(n2 > 0.0)) {
#pragma unroll
        for (int i = 0; i < 8; ++i) dg[i] = 0;
        branch[r * (pd / 8) + off / 8 + blk] = 0;
        return;
    }
    const double inv = 1.0 / sqrt(n2);
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float u = static_cast<float>(static_cast<double>(rr[r * pd + off + blk * 8 + i]) * inv);
        v[i] = static_cast<double>(u) * srd;
    }
    uint16_t out[8];
    const int br = encode_block(v, et, out);
#pragma unroll
    for (int i = 0; i < 8; ++i) dg[i] = out[i];
    branch[r * (pd / 8) + off / 8 + blk] = static_cast<uint8_t>(br);
}

// Export: decode every padded slot back to digits/branch, cluster-major
// compact order (positions of padding lanes are skipped).
__global__ void decode_kernel(DevIndex ix, int ntiles, const uint32_t* __restrict__ list_of_tile,
                              const uint64_t* __restrict__ list_begin, uint16_t* __restrict__ digits,
                              uint8_t* __restrict__ branch) {
    const size_t e = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t total = static_cast<size_t>(ntiles) * 32 * ix.B;
    if (e >= total) return;
    const size_t slot = e / ix.B;
    const int blk = static_cast<int>(e - slot * ix.B);
    const int tile = static_cast<int>(slot / 32), lane = static_cast<int>(slot % 32);
    const uint32_t list = list_of_tile[tile];
    const uint32_t local = (tile - ix.tile_begin[list]) * 32 + lane;
    if (local >= ix.list_len[list]) return;
    const size_t pos = list_begin[list] + local;
    const int off = blk * 8 * ix.bits;
    uint32_t w[5];
    for (int j = 0; j < 5; ++j) {
        const int wi = (off >> 5) + j;
        const int c = wi >> 2;
        if (c < ix.nch) {
            const uint4 v = ix.codes[(static_cast<size_t>(tile) * ix.nch + c) * 32 + lane];
            const uint32_t arr[4] = {v.x, v.y, v.z, v.w};
            w[j] = arr[wi & 3];
        } else {
            w[j] = 0;
        }
    }
    const int bits = ix.bits;
    const int base = off & 31;
    uint32_t par = 0, dg[8];
    for (int i = 0; i < 7; ++i) {
        dg[i] = field(w, base + i * bits, bits);
        par ^= dg[i];
    }
    const uint32_t f7 = field(w, base + 7 * bits, bits);
    dg[7] = (f7 & ~1u) | (par & 1u);
    for (int i = 0; i < 8; ++i) digits[(pos * ix.B + blk) * 8 + i] = static_cast<uint16_t>(dg[i]);
    branch[pos * ix.B + blk] = static_cast<uint8_t>(f7 & 1u);
}

int trunc_dim(int dim) {
    int td = 1;
    while ((td << 1) <= dim) td <<= 1;
    return td;
}

}  // namespace

int launch_mean(const float* x, size_t n, int dim, float* mu_out, cudaStream_t s) {
    mean_kernel<<<(dim + 63) / 64, 64, 0, s>>>(x, n, dim, mu_out);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_centroids(const uint8_t* signs, int dim, int pd, const float* cen_raw, int nlist,
                     const float* mean_rot, float* cen_rot, float* cn2, cudaStream_t s) {
    const int td = trunc_dim(dim);
    const float fac = 1.0f / sqrtf(static_cast<float>(td));
    centroids_kernel<<<nlist, 256, pd * sizeof(float), s>>>(signs, dim, pd, td, fac, cen_raw, mean_rot,
                                                             cen_rot, cn2);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

static size_t build_smem(int rb, int pd, int B, int nch) { return BuildSmem(rb, pd, B, nch).total; }

int launch_build_encode(const DevIndex& ix, const DevEncTables& et, const BuildEncodeArgs& a,
                        uint4* codes, float* g1, float* h3, cudaStream_t s) {
    int rb = 16;
    while (rb > 1 && build_smem(rb, ix.pd, ix.B, ix.nch) > 160 * 1024) rb >>= 1;
    const size_t smem = build_smem(rb, ix.pd, ix.B, ix.nch);
    if (smem > 200 * 1024) fail(E8QC_EINVAL, "padded_dim too large for the build kernel");
    E8QC_CUDA(cudaFuncSetAttribute(build_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(smem)));
    const int td = trunc_dim(ix.dim);
    const float fac = 1.0f / sqrtf(static_cast<float>(td));
    const int grid = a.ntiles * (32 / rb);
    if (grid > 0)
        build_encode_kernel<<<grid, kBuildThreads, smem, s>>>(ix, et, a, rb, td, fac, codes, g1, h3);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_encode(const DevEncTables& et, const float* unit, size_t n, int pd, double srd,
                  uint16_t* digits, uint8_t* branch, cudaStream_t s) {
    const size_t total = n * static_cast<size_t>(pd / 8);
    if (total == 0) return 0;
    encode_kernel<<<static_cast<unsigned>((total + 127) / 128), 128, 0, s>>>(et, unit, n, pd, srd, digits,
                                                                              branch);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_me8q_encode(const DevEncTables& et, const float* rr, int pd, const double* norm2, int ncoded, int run,
                       int off, int len, size_t n, double srd, uint16_t* digits, uint8_t* branch, cudaStream_t s) {
    const size_t total = n * static_cast<size_t>(len / 8);
    if (total == 0) return 0;
    me8q_encode_kernel<<<static_cast<unsigned>((total + 127) / 128), 128, 0, s>>>(et, rr, pd, norm2, ncoded, run, off,
                                                                                   len, n, srd, digits, branch);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_decode(const DevIndex& ix, int ntiles, const uint32_t* list_of_tile,
                       const uint64_t* list_begin, uint16_t* digits, uint8_t* branch,
                       cudaStream_t s) {
    const size_t total = static_cast<size_t>(ntiles) * 32 * ix.B;
    if (total == 0) return 0;
    decode_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(ix, ntiles, list_of_tile,
                                                                              list_begin, digits, branch);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

}  // namespace e8qc
