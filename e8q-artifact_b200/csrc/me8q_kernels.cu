// ME8Q build and single-vector kernels (layout in me8q.h).
//
// Build per chunk of rows: prep (residual to the list centroid, per-run
// FHT-Kac-4 rotation in shared memory, fp64 norms) -> the E8Q block encoder
// per coded run (build_kernels.cu) -> fits and packing. Every sum the
// reference accumulates sequentially (src/index/me8q_build.cpp:203-309,
// src/quantization/me8q_codec.cpp:149-167, src/index/me8q_common.cpp:11-35)
// is accumulated here by one thread in the same order, with the reference
// build's fused multiply-adds, so codes and (coef, h2) come out bit-identical.
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "internal.h"
#include "me8q.h"
#include "me8q_stream.cuh"

namespace e8qc {

namespace {

__global__ void variance_kernel(const float* __restrict__ x, size_t n, int dim, float* __restrict__ var) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= dim) return;
    float mean = 0.0f;
    for (size_t i = 0; i < n; ++i) mean = __fadd_rn(mean, x[i * dim + j]);
    mean = __fdiv_rn(mean, static_cast<float>(n));
    double t = 0.0;
    for (size_t i = 0; i < n; ++i) {
        const double d = static_cast<double>(x[i * dim + j]) - static_cast<double>(mean);
        t = __fma_rn(d, d, t);
    }
    var[j] = static_cast<float>(t / static_cast<double>(n));
}

// One CTA per row (see launch_me8q_prep).
__global__ void prep_kernel(const float* __restrict__ x, size_t ld, int dim, int pd, const float* __restrict__ cen_pad,
                            const uint32_t* __restrict__ cid, Me8qView v, size_t row0, float* __restrict__ rr,
                            double* __restrict__ norm2, double* __restrict__ drop) {
    extern __shared__ float psx[];
    float* sx = psx;       // unrotated residual
    float* sr = psx + pd;  // rotated runs
    const size_t r = blockIdx.x, grow = row0 + r;
    const float* cen = cen_pad ? cen_pad + static_cast<size_t>(cid[grow]) * pd : nullptr;
    for (int i = threadIdx.x; i < pd; i += blockDim.x) {
        float val = 0.0f;
        if (i < dim) val = cen ? __fsub_rn(x[grow * ld + i], cen[i]) : x[grow * ld + i];
        sx[i] = val;
        sr[i] = val;
    }
    __syncthreads();
    for (int q = 0; q < v.nruns; ++q) {
        const Me8qRun run = v.runs[q];
        if (run.bits == 0) continue;
        rotate_rows_smem(sr + run.off, 1, run.len, run.len, run.td, run.fac, v.signs + run.soff);
    }
    for (int q = 0; q < v.nruns; ++q) {
        const Me8qRun run = v.runs[q];
        if (run.bits != 0) continue;
        for (int i = threadIdx.x; i < run.len; i += blockDim.x) sr[run.off + i] = 0.0f;
    }
    __syncthreads();
    if (norm2 && static_cast<int>(threadIdx.x) < v.nruns) {
        const Me8qRun run = v.runs[threadIdx.x];
        if (run.bits != 0) {
            double s = 0.0;
            for (int j = 0; j < run.len; ++j) {
                const double a = static_cast<double>(sr[run.off + j]);
                s = __fma_rn(a, a, s);
            }
            norm2[r * v.ncoded + run.coded] = s;
        }
    }
    if (drop && threadIdx.x == blockDim.x - 1) {
        double s = 0.0;
        for (int q = 0; q < v.nruns; ++q) {
            const Me8qRun run = v.runs[q];
            if (run.bits != 0) continue;
            for (int j = 0; j < run.len; ++j) {
                const double a = static_cast<double>(sx[run.off + j]);
                s = __fma_rn(a, a, s);
            }
        }
        drop[r] = s;
    }
    for (int i = threadIdx.x; i < pd; i += blockDim.x) rr[r * pd + i] = sr[i];
}

// One thread per (row, coded run): the run's fits (ScoreVectorCode) from its
// digits, (coef, h2), and its words of the row's stream.
__global__ void fits_pack_kernel(Me8qView v, const float* __restrict__ rr, const uint16_t* __restrict__ digits,
                                 const uint8_t* __restrict__ branch, const double* __restrict__ norm2,
                                 const double* __restrict__ drop, const uint32_t* __restrict__ cid,
                                 const float* __restrict__ cen_rot, int pd, size_t row0, size_t n,
                                 const uint32_t* __restrict__ slot_of_row, int drop_energy, uint4* codes,
                                 float* __restrict__ coef, float* __restrict__ h2o) {
    const size_t t = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n * static_cast<size_t>(v.ncoded)) return;
    const size_t r = t / v.ncoded;
    const int s = static_cast<int>(t - r * v.ncoded);
    Me8qRun run{};
    for (int q = 0; q < v.nruns; ++q)
        if (v.runs[q].coded == s) run = v.runs[q];
    const size_t grow = row0 + r;
    const size_t slot = slot_of_row[grow];
    const uint32_t c = cid[grow];
    const int b = run.bits, Qb = 1 << b;
    const float* lev0 = v.levels + v.chunks[run.off / 64].lev;
    const uint16_t* dg = digits + r * pd + run.off;
    const uint8_t* br = branch + r * (pd / 8) + run.off / 8;
    const float* x = rr + r * pd + run.off;
    const float* cr = cen_rot + static_cast<size_t>(c) * pd + run.off;
    double dot_r = 0.0, dot_c = 0.0;
    for (int blk = 0; blk < run.len / 8; ++blk) {
        const float* lv = lev0 + (br[blk] ? Qb : 0);
        for (int i = 0; i < 8; ++i) {
            const double l = static_cast<double>(lv[dg[blk * 8 + i]]);
            dot_r = __fma_rn(static_cast<double>(x[blk * 8 + i]), l, dot_r);
            dot_c = __fma_rn(static_cast<double>(cr[blk * 8 + i]), l, dot_c);
        }
    }
    const double n2 = norm2[r * v.ncoded + s];
    double cf = dot_r > 1e-12 ? n2 / dot_r : 0.0;
    if (!isfinite(cf)) cf = 0.0;
    double hh = __fma_rn(2.0 * cf, dot_c, n2);
    if (drop_energy && s == v.ncoded - 1) hh += drop[r];
    coef[static_cast<size_t>(s) * v.nslots + slot] = static_cast<float>(cf);
    h2o[static_cast<size_t>(s) * v.nslots + slot] = static_cast<float>(isfinite(hh) ? hh : 0.0);
    // stream words of this run: block j at bit j*8b, digit i at +i*b, digit 7
    // with the branch in its lowest bit
    const int nch = v.base.nch;
    unsigned long long acc = 0;
    int fill = 0, w = run.word0;
    for (int blk = 0; blk < run.len / 8; ++blk) {
        for (int i = 0; i < 8; ++i) {
            uint32_t f = dg[blk * 8 + i];
            if (i == 7) f = (f & ~1u) | (br[blk] & 1u);
            acc |= static_cast<unsigned long long>(f) << fill;
            fill += b;
            if (fill >= 32) {
                *me8q_word_ptr(codes, nch, slot, w++) = static_cast<uint32_t>(acc);
                acc >>= 32;
                fill -= 32;
            }
        }
    }
}

__global__ void hsum_kernel(Me8qView v, float* __restrict__ hsum) {
    const size_t slot = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (slot >= v.nslots) return;
    double s = 0.0;
    for (int q = 0; q < v.ncoded; ++q) s += static_cast<double>(v.h2[static_cast<size_t>(q) * v.nslots + slot]);
    hsum[slot] = static_cast<float>(s);
}

__global__ void estimate_kernel(Me8qView v, const float* __restrict__ rq, const float* __restrict__ qpad,
                                const float* __restrict__ cen_pad, uint32_t list, uint32_t slot, float* out) {
    const int pd = v.base.pd;
    double d2 = 0.0;
    for (int j = 0; j < pd; ++j) {
        const double d = static_cast<double>(qpad[j]) - static_cast<double>(cen_pad[static_cast<size_t>(list) * pd + j]);
        d2 = __fma_rn(d, d, d2);
    }
    double acc = d2;
    for (int q = 0; q < v.nruns; ++q) {
        const Me8qRun run = v.runs[q];
        if (run.bits == 0) continue;
        const double cf = v.coef[static_cast<size_t>(run.coded) * v.nslots + slot];
        const double hh = v.h2[static_cast<size_t>(run.coded) * v.nslots + slot];
        if (cf == 0.0) {
            acc += hh;
            continue;
        }
        const float* lev0 = v.levels + v.chunks[run.off / 64].lev;
        float sc = 0.0f;
        for (int j = 0; j < run.len / 8; ++j) {
            uint32_t dg[8];
            const int br = me8q_block(v.base.codes, v.base.nch, slot, run.word0, run.bits, j, dg);
            const float* lv = lev0 + (br ? (1 << run.bits) : 0);
            for (int i = 0; i < 8; ++i) sc = __fmaf_rn(rq[run.off + j * 8 + i], lv[dg[i]], sc);
        }
        acc += __fma_rn(-2.0 * cf, static_cast<double>(sc), hh);
    }
    *out = static_cast<float>(acc);
}

__global__ void decode_kernel(Me8qView v, int ntiles, const uint32_t* __restrict__ list_of_tile,
                              const uint64_t* __restrict__ list_begin, int pd, uint16_t* __restrict__ digits,
                              uint8_t* __restrict__ branch) {
    const size_t slot = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (slot >= static_cast<size_t>(ntiles) * 32) return;
    const uint32_t tile = static_cast<uint32_t>(slot >> 5);
    const uint32_t L = list_of_tile[tile];
    const uint32_t local = static_cast<uint32_t>(slot - static_cast<size_t>(v.base.tile_begin[L]) * 32);
    if (local >= v.base.list_len[L]) return;
    const size_t pos = list_begin[L] + local;
    for (int q = 0; q < v.nruns; ++q) {
        const Me8qRun run = v.runs[q];
        for (int j = 0; j < run.len / 8; ++j) {
            uint32_t dg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            int br = 0;
            if (run.bits != 0) br = me8q_block(v.base.codes, v.base.nch, slot, run.word0, run.bits, j, dg);
            for (int i = 0; i < 8; ++i) digits[pos * pd + run.off + j * 8 + i] = static_cast<uint16_t>(dg[i]);
            branch[pos * (pd / 8) + run.off / 8 + j] = static_cast<uint8_t>(br);
        }
    }
}

// ME8Q proxy plane, the int8 operand of the precision scan (the E8Q proxy
// plane's layout: slot s, dimension i at (s/8)*8*pd + (i/16)*128 + (s%8)*16 +
// i%16). Per slot the decoded levels scaled by the slot's coef of their run,
// L' = coef_s * level, are quantised with one scale per slot: p = rint(L' /
// sigma), sigma = max|L'| / 127 (0 when every L' is 0), so sigma * p ~ L' and
// one int8 contraction over all runs approximates sum_s coef_s * S_s. One
// thread per slot: pass 1 finds max|L'|, pass 2 writes 16 proxies per 16-byte
// store. Dropped runs and padding slots are zero.
__global__ void proxy_kernel(Me8qView v, int nslots, unsigned char* __restrict__ plane, float* __restrict__ sigma) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslots) return;
    const int pd = v.base.pd, nch = v.base.nch;
    const uint32_t L = v.base.list_of_tile[slot >> 5];
    const bool live = static_cast<uint32_t>(slot) - v.base.tile_begin[L] * 32u < v.base.list_len[L];
    float amax = 0.0f;
    if (live) {
        for (int q = 0; q < v.nruns; ++q) {
            const Me8qRun run = v.runs[q];
            if (run.bits == 0) continue;
            const float cf = v.coef[static_cast<size_t>(run.coded) * v.nslots + slot];
            if (cf == 0.0f) continue;
            const float* lev0 = v.levels + v.chunks[run.off / 64].lev;
            for (int j = 0; j < run.len / 8; ++j) {
                uint32_t dg[8];
                const int br = me8q_block(v.base.codes, nch, slot, run.word0, run.bits, j, dg);
                const float* lv = lev0 + (br ? (1 << run.bits) : 0);
                for (int i = 0; i < 8; ++i) amax = fmaxf(amax, fabsf(__fmul_rn(cf, __ldg(lv + dg[i]))));
            }
        }
    }
    const float inv = amax > 0.0f ? 127.0f / amax : 0.0f;
    sigma[slot] = amax > 0.0f ? amax / 127.0f : 0.0f;
    unsigned char* dst = plane + static_cast<size_t>(slot >> 3) * 8 * pd + (slot & 7) * 16;
    for (int q = 0; q < v.nruns; ++q) {
        const Me8qRun run = v.runs[q];
        const float cf = (live && run.bits != 0) ? v.coef[static_cast<size_t>(run.coded) * v.nslots + slot] : 0.0f;
        const float* lev0 = run.bits != 0 && run.off < v.route_dim ? v.levels + v.chunks[run.off / 64].lev : v.levels;
        for (int g = 0; g < run.len / 16; ++g) {
            uint32_t o[4] = {0u, 0u, 0u, 0u};
            if (cf != 0.0f) {
                for (int h = 0; h < 2; ++h) {
                    uint32_t dg[8];
                    const int br = me8q_block(v.base.codes, nch, slot, run.word0, run.bits, 2 * g + h, dg);
                    const float* lv = lev0 + (br ? (1 << run.bits) : 0);
                    for (int i = 0; i < 8; ++i) {
                        int p = __float2int_rn(__fmul_rn(__fmul_rn(cf, __ldg(lv + dg[i])), inv));
                        p = p > 127 ? 127 : (p < -127 ? -127 : p);
                        const int e = h * 8 + i;
                        o[e >> 2] |= (static_cast<uint32_t>(p) & 0xFFu) << (8 * (e & 3));
                    }
                }
            }
            *reinterpret_cast<uint4*>(dst + static_cast<size_t>(run.off / 16 + g) * 128) =
                make_uint4(o[0], o[1], o[2], o[3]);
        }
    }
}

}  // namespace

int launch_me8q_proxy(const Me8qView& v, int ntiles, unsigned char* plane, float* sigma, cudaStream_t s) {
    const int nslots = ntiles * 32;
    if (nslots == 0) return 0;
    proxy_kernel<<<(nslots + 127) / 128, 128, 0, s>>>(v, nslots, plane, sigma);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_me8q_variance(const float* x, size_t n, int dim, float* var, cudaStream_t s) {
    variance_kernel<<<(dim + 127) / 128, 128, 0, s>>>(x, n, dim, var);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_me8q_prep(const float* x, size_t ld, int dim, int pd, const float* cen_pad, const uint32_t* cid,
                     const Me8qView& v, size_t row0, size_t n, float* rr, double* norm2, double* drop,
                     cudaStream_t s) {
    if (n == 0) return 0;
    const size_t smem = static_cast<size_t>(2) * pd * sizeof(float);
    if (smem > 48 * 1024) {
        static size_t configured[64] = {};
        int dev = 0;
        E8QC_CUDA(cudaGetDevice(&dev));
        if (configured[dev & 63] < smem) {
            E8QC_CUDA(cudaFuncSetAttribute(prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem)));
            configured[dev & 63] = smem;
        }
    }
    prep_kernel<<<static_cast<unsigned>(n), 256, smem, s>>>(x, ld, dim, pd, cen_pad, cid, v, row0, rr, norm2, drop);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_me8q_fits_pack(const Me8qView& v, const float* rr, const uint16_t* digits, const uint8_t* branch,
                          const double* norm2, const double* drop, const uint32_t* cid, const float* cen_rot,
                          int pd, size_t row0, size_t n, const uint32_t* slot_of_row, bool drop_energy,
                          uint4* codes, float* coef, float* h2, cudaStream_t s) {
    const size_t total = n * static_cast<size_t>(v.ncoded);
    if (total == 0) return 0;
    fits_pack_kernel<<<static_cast<unsigned>((total + 127) / 128), 128, 0, s>>>(
        v, rr, digits, branch, norm2, drop, cid, cen_rot, pd, row0, n, slot_of_row, drop_energy ? 1 : 0, codes, coef,
        h2);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_me8q_hsum(const Me8qView& v, float* hsum, cudaStream_t s) {
    if (v.nslots == 0) return 0;
    hsum_kernel<<<static_cast<unsigned>((v.nslots + 255) / 256), 256, 0, s>>>(v, hsum);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_me8q_estimate(const Me8qView& v, const float* rq, const float* qpad, const float* cen_pad,
                         uint32_t list, uint32_t slot, float* out, cudaStream_t s) {
    estimate_kernel<<<1, 1, 0, s>>>(v, rq, qpad, cen_pad, list, slot, out);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

int launch_me8q_decode(const Me8qView& v, int ntiles, const uint32_t* list_of_tile, const uint64_t* list_begin,
                       int pd, uint16_t* digits, uint8_t* branch, cudaStream_t s) {
    const size_t total = static_cast<size_t>(ntiles) * 32;
    if (total == 0) return 0;
    decode_kernel<<<static_cast<unsigned>((total + 127) / 128), 128, 0, s>>>(v, ntiles, list_of_tile, list_begin, pd,
                                                                             digits, branch);
    E8QC_CUDA(cudaGetLastError());
    return 1;
}

}  // namespace e8qc
