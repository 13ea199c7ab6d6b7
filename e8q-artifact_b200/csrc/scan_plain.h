// Plain-scan launch geometry shared by the host and the kernel.
#pragma once

#include <stddef.h>

#include "internal.h"

namespace e8qc {

// Copies of the [2][2^bits] level table kept in shared memory: one per lane
// (bank-conflict-free gathers) while the copies fit 32 KB, fewer above.
__host__ __device__ constexpr int table_rep(int bits) {
    return (8192 >> (bits + 1)) >= 32 ? 32 : ((8192 >> (bits + 1)) >= 1 ? (8192 >> (bits + 1)) : 1);
}

// Launch geometry of the plain scan: warps per CTA, vectors per lane of a
// work unit (1 or 2), tiles per batch and the dynamic shared memory (query,
// tile offsets, the batch's unit partial sums, merge buffers; the level table
// copies too for the rates that do not fit the static table).
struct ScanGeo {
    int warps;
    int v;
    int tb_tiles;
    size_t smem;
};

// max_tiles_per_cta: the most tiles any CTA of the launch can get.
ScanGeo plain_scan_geo(const DevIndex& ix, size_t max_tiles_per_cta);
size_t scan_smem_bytes(const DevIndex& ix, int tb_tiles, int v);
int launch_scan_plain(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k,
                      const ScanWork& sw, const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s);

}  // namespace e8qc
