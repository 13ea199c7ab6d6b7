// Precision search path (precision.cu): INT8 tensor-core candidate generation
// followed by exact rescoring of each query's candidates.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "internal.h"
#include "workspace.h"

namespace e8qc {

// The int8 step of the E8Q proxy plane for `bits` at padded dimension pd
// (set as DevIndex::proxy_scale once the plane is built).
float precision_proxy_step(int bits, int pd);

// Bytes of the int8 proxy plane: the padded slots (plus one MMA tile of 256
// slots read past the last list) x pd.
size_t proxy_plane_bytes(const DevIndex& ix, size_t ntiles);

// Decode every slot's code into the proxy plane (layout in precision.cu).
int launch_build_proxy(const DevIndex& ix, int ntiles, uint4* plane, cudaStream_t s);

// Slot-major copy of an E8Q index's codes (each slot's nch chunks
// contiguous), read by the exact rescoring of the precision mode.
size_t vcodes_bytes(const DevIndex& ix, size_t ntiles);
int launch_vcodes(const DevIndex& ix, int ntiles, uint4* out, cudaStream_t s);

// A row-group int8 plane (8-row groups of 16-byte core-matrix rows, K-major:
// row r, byte k at (r/8)*8*pd + (k/16)*128 + (r%8)*16 + k%16) as a 2D tensor
// map over row groups (8*pd bytes each, seen as 2*pd u32) whose box is
// box_rows row groups x box_u32 u32 (128 u32: one 64-byte K-chunk of each row;
// 64 u32: a 32-byte one).
CUtensorMap plane_map(const void* base, size_t row_groups, int pd, uint32_t box_rows, uint32_t box_u32 = 128);

// Candidates kept per query for exact rescoring at a given k.
int precision_candidates(int k);

// Search nq rotated queries; same argument meaning as batched_search.
// rows_per_query bounds the vectors one query's probes can reach (the padded
// slots of the nprobe longest lists): the proxy scratch of a chunk of queries
// is sized from it, and batches whose scratch would exceed 2 GiB run in chunks.
// me8q: the ME8Q index whose view `ix` is (its proxy plane in ix.proxy, the
// per-slot proxy scale in ix.g1, hsum in ix.h3): slot-scaled level proxies and
// the ME8Q estimator for rescoring. NULL for an E8Q index.
// Device bytes of the proxy-distance rows one ragged call of nq queries
// holds at once (it runs in chunks of queries within a fixed budget).
size_t precision_row_scratch(size_t nq, size_t rows_per_query);

struct Me8qView;
int precision_search(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                     const uint32_t* np_arr, size_t k, size_t nprobe, size_t out_stride, uint32_t* out_ids,
                     float* out_d, size_t rows_per_query, cudaStream_t s, const Me8qView* me8q = nullptr);

}  // namespace e8qc
