// Batch routing keys on the int8 tensor cores (route_tc.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "internal.h"
#include "workspace.h"

namespace e8qc {

// Batches from this many queries compute their routing keys with
// route_tc_keys (below it the fp64 route GEMM is as fast).
constexpr size_t kRouteTcMinQueries = 256;

// Whether route_tc_keys serves this index and batch size (at most 25600
// lists, padded dimension at most 4096).
bool route_tc_applies(const DevIndex& ix, size_t nq);

// The (query, list) key matrix of nq rotated queries in ws.b_keys, equal to
// the fp64 route GEMM's except where the tensor-core bound cannot settle a
// key: there the key holds a lower bound of the d2 bits with bit 31 of its low
// word set and ws.r_ub an upper bound (select_kernel resolves those that
// matter). Needs ws.b_qn2 (the queries' squared norms). Returns the kernels
// launched.
int route_tc_keys(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, cudaStream_t s);

}  // namespace e8qc
