// The reference's E8Q index file (E8AX) read into host arrays laid out the
// way this library's device index holds them (io_e8ax.cpp).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <vector>

#include "internal.h"

namespace e8qc {

struct E8axParts {
    size_t n = 0, dim = 0, nlist = 0, pd = 0, ntiles = 0;
    int bits = 0, nch = 0;
    float prune_alpha = 1.0f;
    std::vector<uint8_t> signs;          // rotator sign bytes
    std::vector<float> mean_rot;         // pd
    std::vector<float> cen_rot, cn2;     // nlist x pd, nlist
    std::vector<uint64_t> list_begin;    // nlist + 1, cluster-major offsets
    std::vector<uint32_t> tile_begin;    // nlist + 1
    std::vector<uint32_t> ids_compact;   // n, cluster-major global ids
    std::vector<uint32_t> slot_ids;      // ntiles * 32 (UINT32_MAX on padding)
    std::vector<float> g1, h3;           // ntiles * 32
    std::vector<uint4> codes;            // ntiles * nch * 32: chunk c of lane l at [tile][c][l]
};

// Throws Error(E8QC_EIO) for an unreadable, foreign or inconsistent file.
// sign_bytes_for_dim: the rotator's sign-byte count for a dimension.
E8axParts read_e8ax(const char* path, size_t sign_bytes_for_dim(size_t));

}  // namespace e8qc
