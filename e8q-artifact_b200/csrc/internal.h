// Internal declarations shared by the host code and the CUDA kernels of
// libe8qcuda.so. Not installed; the public surface is include/e8qc.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "e8qc.h"

namespace e8qc {

constexpr int kMaxBits = 13;
constexpr int kMaxK = 128;
constexpr int kTile = 32;  // vectors per tile: one warp lane per vector

// Library error: carries an e8qc status code to the C boundary.
struct Error {
    int code;
    std::string msg;
};
[[noreturn]] void fail(int code, const std::string& msg);
// A checked host-allocation point: throws std::bad_alloc while injected
// failures (e8qc_debug_fail_host_allocs) remain, consuming one.
void host_alloc_point();
void cuda_check(cudaError_t e, const char* what);
#define E8QC_CUDA(x) ::e8qc::cuda_check((x), #x)

// ---------------------------------------------------------------------------
// Codec constants (host). Restated from the reference codec
// (src/quantization/e8q_codec.cpp); see codec_host.cpp.
double inv_normal_cdf(double p);
std::vector<double> branch_levels(int bits, int branch);
double fixed_scale(int bits);
// PhiInv by Newton steps on Phi, and the per-query concentration quantile
// lambda = max(1, PhiInv(1 - min(alpha / k_eff, 0.49)))
// (src/index/e8q_internal.hpp:75-107).
double phi_inv(double p);
float ortho_quantile(double alpha, size_t k_eff);
constexpr double kSigmaC = 1.1180339887498949;

// Sorted level table with the bounded-bin insertion index
// (src/quantization/e8q_codec.cpp:70-123): merged four-class table when it
// alternates, else four per-(branch, parity) tables.
struct LevelTableHost {
    std::vector<double> lev;   // pad x -inf | n levels | pad x +inf
    std::vector<uint16_t> dig; // same indexing
    std::vector<uint32_t> bin_lo;
    int pad = 0;
    int n = 0;
    double bin_lo_v = 0.0, bin_scale = 0.0;
    int nbins = 1;
    int usable = 0;
};

struct EncTablesHost {
    int bits = 0;
    int alternating = 0;
    LevelTableHost merged;
    LevelTableHost parity[2][2];  // [branch][odd]
    std::vector<double> levels[2];
};
const EncTablesHost& enc_tables_host(int bits);

// Device view of one level table.
struct DevLevelTable {
    const double* lev;      // points at the first real level (pads around it)
    const uint16_t* dig;    // same indexing as lev
    const uint32_t* bin_lo;
    int n, nbins, usable;
    double bin_lo_v, bin_scale;
};

struct DevEncTables {
    int bits, alternating;
    DevLevelTable merged;
    DevLevelTable parity[4];  // [branch*2 + odd]
    const double* levels[2];  // 2^bits each
};
// Per (device, bits) upload, cached for the process lifetime.
const DevEncTables& enc_tables_device(int device, int bits);

// ---------------------------------------------------------------------------
// Device index layout.
//
// Vectors are stored list-major ("cluster-major"), each list padded to whole
// tiles of 32 vectors. A vector's code is a little-endian bitstream of B =
// padded_dim/8 blocks of 8*bits bits; inside a block digit i occupies bits
// [i*bits, (i+1)*bits) except that the lowest bit of digit 7 holds the branch
// (digit 7's own LSB is the parity of digits 0..6, the E8 quotient-shell
// constraint, so it is not stored). The stream is padded to whole 16-byte
// chunks (nch per vector), and a tile stores chunk c of lane l at
// [tile][c][l] so a warp reading chunk c touches 512 contiguous bytes.
struct DevIndex {
    int dim, pd, B, bits, nlist, nch;
    int ntiles;                  // 32-slot tiles over all lists
    const uint8_t* signs;        // 4*pd/8 rotation sign bits
    const float* mean_rot;       // pd
    const float* cen;            // nlist*pd rotated, centred centroids
    const float* cn2;            // nlist squared norms
    const uint32_t* tile_begin;  // nlist+1
    const uint32_t* list_len;    // nlist vectors per list
    const uint4* codes;          // ntiles*nch*32 chunks
    const float* g1;             // ntiles*32
    const float* h3;             // ntiles*32
    const uint32_t* ids;         // ntiles*32, UINT32_MAX on padding lanes
    const float* tab;            // [2][2^bits] level/sqrt(pd) refine tables
    const uint32_t* list_order;  // 2 x nlist list ids: longest list first, then list id order
    const uint32_t* list_of_tile;  // ntiles: the list each tile belongs to
    const uint4* proxy;            // precision mode's int8 proxy plane, or NULL until built
    float proxy_scale;             // E8Q: the plane's level step (proxy * step ~ table level)
    const uint4* vcodes;           // precision mode: the codes slot-major (nch chunks per slot), or NULL
};

inline int code_chunks(int pd, int bits) { return (pd / 8 * 8 * bits + 127) / 128; }

// ---------------------------------------------------------------------------
// Kernel launchers (each returns the number of kernels it launched).

// Rotation + mean-centring of nq queries: out[nq][pd] = rot(q) - mean_rot.
int launch_rotate(const DevIndex& ix, const float* q, int nq, float* out, cudaStream_t s);
// nq synthetic rotated queries near the index's lists (tuning runs).
int launch_synth_queries(const DevIndex& ix, int nq, unsigned long long seed, float* out, cudaStream_t s);
// Raw rotation (no centring): n rows of dim floats -> n rows of pd floats.
int launch_rotate_raw(const uint8_t* signs, int dim, int pd, const float* src, int n, float* dst,
                      const float* subtract, cudaStream_t s);

struct RouteWork {
    uint64_t* keys;        // nlist
    uint32_t* probes;      // nlist (first nprobe used)
    float* probe_d2;       // nlist
    uint32_t* tile_off;    // nlist+1 exclusive prefix of probed tiles
    uint32_t* counter;     // last-CTA-done counter (self-resetting)
    uint32_t* total_tiles; // 1
    uint2* probe_info;     // nlist: (first tile, vectors) of the p-th probed list
};
// One query: d2 to every centroid, then (last CTA) the nprobe nearest lists
// and the prefix of their tile counts.
int launch_route_one(const DevIndex& ix, const float* rq, int nprobe, const RouteWork& w,
                     cudaStream_t s);

struct ScanWork {
    float* part_d;      // grid*kmax
    uint32_t* part_id;  // grid*kmax
    uint32_t* counter;  // self-resetting
    uint32_t* err;      // device error word (bounded waits that gave up)
    int grid;
    uint32_t stuck_ms = 0;  // test hook: CTA 0 waits this long on a barrier nothing completes
};

// Build kernels.
int launch_mean(const float* x, size_t n, int dim, float* mu_out, cudaStream_t s);
int launch_centroids(const uint8_t* signs, int dim, int pd, const float* cen_raw, int nlist,
                     const float* mean_rot, float* cen_rot, float* cn2, cudaStream_t s);
struct BuildEncodeArgs {
    const float* base;       // n*dim raw rows (device)
    const uint32_t* row_of;  // ntiles*32 slot -> row id (UINT32_MAX padding)
    const uint32_t* list_of_tile;  // ntiles
    int ntiles;
    double srd;              // FixedScale(bits) * sqrt(pd)
    double inv_level_scale;  // 1/sqrt(pd)
    double w_cls[2];         // branch-averaged level mean of each top-bit class (the scan basis)
    float* ortho;            // ntiles*32*3: per slot the scan-bank inputs (base, weight, perp), or NULL
};
int launch_build_encode(const DevIndex& ix, const DevEncTables& et, const BuildEncodeArgs& a,
                        uint4* codes, float* g1, float* h3, cudaStream_t s);
int launch_encode(const DevEncTables& et, const float* unit, size_t n, int pd, double srd,
                  uint16_t* digits, uint8_t* branch, cudaStream_t s);
// ME8Q: encode one coded run (offset off, len dims) of n rows whose rotated
// residuals are rr (n x pd) with fp64 norms^2 norm2 (n x ncoded, column run);
// srd = FixedScale(bits) * sqrt(len). Writes digits (n x pd) and branch
// (n x pd/8) for the run's dims.
int launch_me8q_encode(const DevEncTables& et, const float* rr, int pd, const double* norm2, int ncoded, int run,
                       int off, int len, size_t n, double srd, uint16_t* digits, uint8_t* branch, cudaStream_t s);
// Decode device codes back to digits/branch (export, tests).
int launch_decode(const DevIndex& ix, int ntiles, const uint32_t* list_of_tile,
                  const uint64_t* list_begin, uint16_t* digits, uint8_t* branch, cudaStream_t s);
// Estimate one stored vector at tile slot `slot` of list `list`.
// ProbeBoundW of m (query, stored vector) pairs (rotated, centred queries rq
// and base rows rx; slot_of UINT32_MAX marks an invalid pair -> NaN).
int launch_probe_bound(const DevIndex& ix, const float* rq, const float* rx, const uint32_t* qsel,
                       const uint32_t* slot_of, const uint32_t* list_of, const double* dlev, const double* mid, int m,
                       int dim, double* out, cudaStream_t s);
int launch_estimate(const DevIndex& ix, const float* rq, int list, uint32_t slot, float* out,
                    cudaStream_t s);

}  // namespace e8qc
