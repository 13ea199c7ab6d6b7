// What a captured plan (plan.cpp) and the serving loop (server.cpp) need from
// an index: its shape, a one-time preparation per mode, the device scratch of
// a ragged batch, and the ragged batch itself enqueued on a stream with a
// caller's workspace. The E8Q index (index.cpp) and the ME8Q index
// (me8q.cpp) each provide one.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <memory>

#include "e8qc.h"
#include "workspace.h"

namespace e8qc {

struct SearchTarget {
    size_t dim = 0, nlist = 0;
    int device = 0;
    virtual ~SearchTarget() = default;
    // Throws E8QC_EINVAL for a mode the index does not serve.
    virtual void check_mode(int mode) const = 0;
    // One-time, synchronised preparation for a mode (e.g. the precision proxy plane).
    virtual void prepare(int mode) = 0;
    // Upper bound of the device scratch of one ragged call of nq queries.
    virtual size_t bytes(int mode, size_t nq, size_t k_max, size_t np_max) const = 0;
    // Ragged search of nq device-resident queries (not rotated) on stream s:
    // no host synchronisation, no index lock, no allocation once ws has been
    // sized by an earlier call of the same shape. Returns kernels launched.
    virtual uint64_t enqueue(Workspace& ws, int mode, const float* q_dev, size_t nq, const uint32_t* k_dev,
                             const uint32_t* np_dev, size_t k_max, size_t np_max, uint32_t* ids_dev, float* d_dev,
                             cudaStream_t s, bool apply_tuned) = 0;
    // Time the tunable settings of one batch shape; leaves the best in ws.
    virtual void autotune(Workspace& ws, int mode, size_t nq, size_t k, size_t np, cudaStream_t s, int* sched,
                          int* stages) = 0;
    // The stored setting of a batch shape (defaults when none) into ws.
    virtual void stored_tuning(Workspace& ws, int mode, size_t nq, size_t np) = 0;
};

// Throw E8QC_ESTATE when the index is not built.
std::shared_ptr<SearchTarget> e8q_target(e8qc_index* x);
std::shared_ptr<SearchTarget> me8q_target(e8qc_me8q* x);

// Captured plan over a target (plan.cpp): graphs for batch sizes 64, 128, ...
// up to max_q, or (exact_size) for max_q alone.
e8qc_plan* plan_make(std::shared_ptr<SearchTarget> t, int mode, size_t max_q, size_t k_max, size_t np_max,
                     bool autotune, bool exact_size = false);
// Enqueue one batch on s (k / nprobe: host arrays of nq entries; queries and
// outputs host or device), then synchronise and report a kernel timeout.
void plan_enqueue(e8qc_plan* P, const float* queries, size_t nq, const uint32_t* k, const uint32_t* nprobe,
                  uint32_t* out_ids, float* out_dists, cudaStream_t s);
void plan_check(e8qc_plan* P, cudaStream_t s);
// Kernels one run of the plan's largest graph launches.
uint64_t plan_kernels(const e8qc_plan* P);
void plan_free(e8qc_plan* P);

}  // namespace e8qc
