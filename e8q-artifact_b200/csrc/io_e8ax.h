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
    std::vector<uint8_t> banks;          // the 128-byte scan-bank header of every 32-vector batch, file order
};

// The 128-byte scan-bank header of one 32-vector batch from its vectors'
// bank inputs (WriteOrthoBanks, src/index/e8q_build.cpp:31-80).
void ortho_banks(const float* base, const float* weight, const float* perp, size_t cnt, uint8_t* hdr);

// Everything an E8AX file holds, in compact (cluster-major) vector order.
struct E8axSave {
    size_t n = 0, dim = 0, nlist = 0, pd = 0;
    int bits = 0;
    float prune_alpha = 1.0f;        // written to the build-options trailer
    const uint8_t* signs = nullptr;  // rotator sign bytes
    size_t sign_bytes = 0;
    const float* mean_rot = nullptr;     // pd
    const float* cen_rot = nullptr;      // nlist x pd
    const float* cn2 = nullptr;          // nlist
    const uint64_t* list_begin = nullptr;  // nlist + 1
    const uint32_t* ids = nullptr;       // n global ids
    const uint16_t* digits = nullptr;    // n x B x 8
    const uint8_t* branch = nullptr;     // n x B
    const float* g1 = nullptr;           // n
    const float* h3 = nullptr;           // n
    const float* ortho = nullptr;        // n x 3 (bank inputs base, weight, perp), or NULL when
    const uint8_t* banks = nullptr;      // ... the headers are given as they were read
};

// Write an E8AX file the reference's E8qIndex::Load reads (E8qIndex::Save,
// src/index/e8q_io.cpp:35-84). Throws Error(E8QC_EIO) on a write failure.
void write_e8ax(const char* path, const E8axSave& w);

// Throws Error(E8QC_EIO) for an unreadable, foreign or inconsistent file.
// sign_bytes_for_dim: the rotator's sign-byte count for a dimension.
E8axParts read_e8ax(const char* path, size_t sign_bytes_for_dim(size_t));

}  // namespace e8qc
