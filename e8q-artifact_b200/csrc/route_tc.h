// Batch routing on the int8 tensor cores with exact fp64 keys (route_tc.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "internal.h"
#include "workspace.h"

namespace e8qc {

// Batches from this many queries route through route_tc (below it the fp64
// route GEMM is as fast).
constexpr size_t kRouteTcMinQueries = 256;

// Whether route_tc serves this index and batch size (at most 4096 lists and a
// padded dimension of at most 4096).
bool route_tc_applies(const DevIndex& ix, size_t nq);

// Probes of nq rotated queries: probes / pd2 ([nq x np_max], list order) and
// the per-list pair counts in ws.b_cnt (zeroed by the caller), bit-identical
// to the fp64 route GEMM + select. Needs ws.b_qn2 (the queries' squared
// norms), uses ws.b_keys as the (query, list) interval matrix. Returns the
// kernels launched.
int route_tc(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* np_arr, int np_max,
             cudaStream_t s);

}  // namespace e8qc
