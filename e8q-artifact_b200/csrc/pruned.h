// The reference's production (pruned) search on the GPU: coarse rowA pass +
// zero-parallel-residual lower bound + exact refine of the survivors, one warp
// per query in the reference's order. See pruned.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace e8qc {

// Bytes of rowA (one byte per 8-dim block, the digits' top bits) per vector,
// padded to whole 16-byte chunks: the coarse plane stores chunk c of lane l
// of a tile at [tile][c][l].
inline int rowa_chunks(int blocks) { return (blocks + 15) / 16; }

struct PrunedWork {
    unsigned long long* stats;   // [0] candidates scanned, [1] survivors refined (accumulated)
    float* thr;                  // per query: the heap's final k-th distance, or NULL
    uint32_t* err;               // device error word
    const uint8_t* banks;        // ntiles * 128: the scan-bank header of every tile
    const uint4* rowa;           // ntiles * nrc * 32 chunks
    int nrc;                     // rowa_chunks(B)
    float z;                     // OrthoQuantile(prune_alpha, max(4k, 32))
    double w_cls0, w_cls1;       // branch-averaged level mean of each top-bit class
    int disable_prune;           // 1: every candidate is refined (the reference's set_disable_prune)
};

// Scratch of the batched form: per-query u8 LUTs (lut8: nq*B*32 bytes) and
// scalars (scal: nq*4); per group of `group` queries the tile offsets (toff:
// group*(np+1)) and every probed row's LUT sum and bound terms (c_acc, c_P,
// c_perp: group*max_tiles*32 each, max_tiles = the most tiles a query's
// probes can hold); out rows of k.
struct PrunedScratch {
    uint8_t* lut8;
    float* scal;
    uint32_t* toff;
    int* c_acc;
    float* c_P;
    float* c_perp;
    size_t max_tiles;
    int group;
    uint32_t* out_ids;
    float* out_d;
};

// Batched form (nq queries, probes / pd2: nq x np from the batched route):
// the LUTs, then per group of queries the tile offsets, the heap-independent
// coarse values of every probed row at full parallelism, and one warp per
// query taking the reference's decisions in its order with its running heap
// from them; pw.thr (if set) gets each query's final k-th distance and
// pw.stats the candidate / survivor counts.
int launch_pruned_batch(const DevIndex& ix, const float* rq, const uint32_t* probes, const float* pd2, int nq, int np,
                        int k, const PrunedWork& pw, const PrunedScratch& sc, cudaStream_t s);
// The coarse plane of every tile from the codes (rowA byte of block b = the
// top bit of each stored digit field, digit i at bit 7 - i).
int launch_build_rowa(const DevIndex& ix, int ntiles, uint4* rowa, cudaStream_t s);
// The 128-byte scan-bank header of every tile from the build's per-slot
// (base, weight, perp) (ortho: ntiles*32*3 floats; padding lanes by ids).
int launch_ortho_banks(const float* ortho, const uint32_t* ids, int ntiles, uint8_t* hdr, cudaStream_t s);

}  // namespace e8qc
