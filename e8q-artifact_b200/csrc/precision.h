// Precision search path (precision.cu): INT8 tensor-core candidate generation
// followed by exact rescoring of each query's candidates.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "internal.h"
#include "workspace.h"

namespace e8qc {

// Slope of the weighted least-squares line level/sqrt(pd) ~ alpha * (t + eta)
// over both branches (weights: the N(0, s^2) density at each level, s the
// rate's encoding scale).
double precision_alpha(int bits, int pd);

// Candidates kept per query for exact rescoring at a given k.
int precision_candidates(int k);

// Search nq rotated queries; same argument meaning as batched_search.
int precision_search(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* k_arr,
                     const uint32_t* np_arr, size_t k, size_t nprobe, size_t out_stride, uint32_t* out_ids,
                     float* out_d, cudaStream_t s);

}  // namespace e8qc
