// ME8Q (mixed-rate E8Q) on the device: plan runs, the index view the
// kernels read, and the launchers (me8q_kernels.cu, batched.cu).
//
// Per vector the code is one bit stream, coded runs back to back in plan
// order (a run of len dims at b bits takes len*b/32 whole words, since len is
// a multiple of 64); inside a run, block j (8 dims) is the 8b-bit field at
// j*8b whose digit i sits at bits i*b and whose digit 7 has the block's
// branch in its lowest bit (the real lowest bit is the parity of digits
// 0..6) -- the E8Q stream layout, per run. Streams are stored like E8Q
// codes: lists padded to 32-vector tiles, 16-byte chunk c of lane l at
// [tile][c][l]. Per slot and coded run s: coef[s][slot]; per slot the sum of
// its runs' h2 (hsum) and, for export, h2[s][slot].
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "internal.h"
#include "workspace.h"

namespace e8qc {

// One plan run as the kernels see it.
struct Me8qRun {
    int off, len, bits;  // dims [off, off + len), bits per dim (0: dropped)
    int coded;           // index among coded runs, -1 when dropped
    int td;              // FHT window of the run's rotator (largest power of 2 <= len)
    float fac;           // 1 / sqrt(td)
    int soff;            // byte offset of the run's rotator signs
    int word0;           // first 32-bit word of the run in a vector's stream
};

// A 64-dim chunk of the coded prefix: its run's rate, coded index, first
// stream word and the offset of its rate's [2][2^b] level table.
struct Me8qChunk {
    int bits, coded, word0, lev;
};

struct Me8qView {
    DevIndex base;             // route / list / id / code fields (tab, g1, h3, proxy unused)
    const float* coef;         // ncoded x nslots
    const float* h2;           // ncoded x nslots
    const float* hsum;         // nslots
    const Me8qRun* runs;       // nruns
    const Me8qChunk* chunks;   // nchunks (coded prefix / 64)
    const float* levels;       // raw level tables, concatenated per rate
    const uint8_t* signs;      // run rotator signs, concatenated
    int nruns, ncoded, nchunks, route_dim;
    size_t nslots;
};

// The fast layout of the production (pruned) search, me8q_fast.cu.
constexpr int kFastMaxRuns = 16;   // coded runs
constexpr int kFastMaxCols = 512;  // coded 8-dim blocks (4,096 coded dims)

// A coded run as the pruned search sees it: dims [off, off + len) at bits
// per digit, its first stream word and level-table offset, its first plane
// column, and the scan basis pbar[0], pbar[1] of its rate (ClassModelOf,
// src/quantization/me8q_codec.cpp:235-262).
struct Me8qFastRun {
    int off, len, bits, word0, lev, blk0;
    float p0, p1;
};

struct Me8qFast {
    int nrun, cols, colw;    // coded runs, plane columns, plane words per lane (ceil(cols / 4))
    const Me8qFastRun* runs;  // nrun
    const uint32_t* plane;    // ntiles x colw x 32 words
    const float* gain;        // nrun x nslots
    const float* vpc;         // nrun x nslots
    const uint8_t* bank;      // ntiles x nrun x 96: base[32], weight[32], perp[32]
    const float* scl;         // ntiles x nrun x 8: (min, step) of base, weight, perp
    const double* rc_n2;      // nlist x nrun: ||centroid slice of the run||^2
};

// Builds the fast layout of a built index (perp: nrun x nslots scratch).
int launch_me8q_fast_build(const Me8qView& v, const Me8qFast& f, uint32_t* plane, float* gain, float* vpc,
                           float* perp, uint8_t* bank, float* scl, double* rc_n2, cudaStream_t s);

// The production search of nq rotated queries (uniform k and nprobe):
// route, per-query select, per-query LUT, the cascade (one warp per query).
int me8q_pruned_search(const Me8qView& v, const Me8qFast& f, Workspace& ws, const float* rq, size_t nq, size_t k,
                       size_t nprobe, float lambda, size_t out_stride, uint32_t* out_ids, float* out_d,
                       cudaStream_t s);

// Per-dimension variance (float mean row by row, fp64 spread; one thread
// per dimension so the sums follow the reference's order).
int launch_me8q_variance(const float* x, size_t n, int dim, float* var, cudaStream_t s);

// Rows -> padded (x - centroid of its list, when cen_pad is given), each
// coded run rotated by its own rotator, dropped dims zero; optionally the
// fp64 norm^2 of every coded run (n x ncoded) and of the unrotated dropped
// dims (n). Rows row0 .. row0+n-1 of x (leading dimension ld).
int launch_me8q_prep(const float* x, size_t ld, int dim, int pd, const float* cen_pad, const uint32_t* cid,
                     const Me8qView& v, size_t row0, size_t n, float* rr, double* norm2, double* drop,
                     cudaStream_t s);

// Fits (coef, h2) and packing of n encoded rows into their slots.
int launch_me8q_fits_pack(const Me8qView& v, const float* rr, const uint16_t* digits, const uint8_t* branch,
                          const double* norm2, const double* drop, const uint32_t* cid, const float* cen_rot,
                          int pd, size_t row0, size_t n, const uint32_t* slot_of_row, bool drop_energy,
                          uint4* codes, float* coef, float* h2, cudaStream_t s);
// hsum[slot] = sum over coded runs of h2 (fp64, in run order).
int launch_me8q_hsum(const Me8qView& v, float* hsum, cudaStream_t s);

// Exact estimate of one stored vector (Me8qIndex::Estimate): fp64 ||q - c||^2
// over the unrotated padded query, per-run fp32 scores, fp64 combination.
int launch_me8q_estimate(const Me8qView& v, const float* rq, const float* qpad, const float* cen_pad,
                         uint32_t list, uint32_t slot, float* out, cudaStream_t s);

// Decode every slot's runs back to digits / branch, cluster-major compact
// order (the order of the index's ids).
int launch_me8q_decode(const Me8qView& v, int ntiles, const uint32_t* list_of_tile, const uint64_t* list_begin,
                       int pd, uint16_t* digits, uint8_t* branch, cudaStream_t s);

// The int8 proxy plane of the precision scan and its per-slot scale sigma
// (plane: proxy_plane_bytes of the view, zeroed by the caller; sigma: ntiles*32).
int launch_me8q_proxy(const Me8qView& v, int ntiles, unsigned char* plane, float* sigma, cudaStream_t s);

// Grouped (batched) exact search of nq rotated queries: route, select,
// group by list, persistent scan, per-query merge (batched.cu).
int me8q_grouped_search(const Me8qView& v, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                        const uint32_t* np_arr, size_t k, size_t nprobe, size_t out_stride, uint32_t* out_ids,
                        float* out_d, cudaStream_t s);

}  // namespace e8qc
