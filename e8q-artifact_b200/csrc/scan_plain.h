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

// A tile (32 vectors) is streamed in segments of U whole chunk-groups; odd
// rates whose block count leaves half a group end with a tail segment.
struct ScanGeo {
    int ng;         // full groups per vector
    int tail;       // 1 when a half-group (8 blocks) follows
    int U;          // groups per segment
    int nseg;       // segments per tile
    int seg_bytes;  // bytes of one ring stage (128-aligned)
    int warps;      // warps per CTA (shared-memory budget)
};

ScanGeo plain_scan_geo(const DevIndex& ix, size_t max_seg_bytes);
size_t scan_smem_bytes(const DevIndex& ix, const ScanGeo& geo);
int launch_scan_plain(const DevIndex& ix, const float* rq, const RouteWork& rw, int nprobe, int k,
                      const ScanWork& sw, const ScanGeo& geo, uint32_t* out_ids, float* out_d, cudaStream_t s);

}  // namespace e8qc
