// Reader of the reference's E8Q index file (E8AX; written by
// E8qIndex::Save, src/index/e8q_io.cpp:35-84; read by E8qIndex::Load,
// :86-211): header, global ids, rotator signs, rotated mean, rotated
// centroids and their norms, list offsets, the scan arena (per 32-vector
// batch: a 128-byte pruning header, then one "rowA" byte per block per lane)
// and the refine arena (per batch: each lane's (b-1)-bit low digit fields,
// then g1[32], h3[32]), and the optional build-options trailer. The codes are
// decoded back to digits/branch (the split decode of src/index/
// e8q_scan.cpp:34-87: digits 0..6 take rowA's bit 7-i as their top bit over
// the field's low bits, digit 7 its parity-derived LSB, the field's bit 0 of
// digit 7 is the branch; b = 1 keeps the whole code in rowA) and repacked
// into this library's per-vector bit streams in 32-vector tiles. The pruning
// headers are not read: the device scans score every candidate exactly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "io_e8ax.h"

namespace e8qc {

namespace {

constexpr uint32_t kE8axMagic = 0x58413845u;  // "E8AX"
constexpr uint32_t kOptMagic = 0x514F5045u;   // "EPOQ": build-options trailer

struct Reader {
    const std::vector<uint8_t>& buf;
    size_t off = 0;
    const uint8_t* take(size_t bytes, const char* what) {
        if (bytes > buf.size() - off) fail(E8QC_EIO, std::string("short read while loading index (") + what + ")");
        const uint8_t* p = buf.data() + off;
        off += bytes;
        return p;
    }
    template <class T>
    T scalar(const char* what) {
        T v;
        std::memcpy(&v, take(sizeof(T), what), sizeof(T));
        return v;
    }
    template <class T>
    std::vector<T> array(size_t count, const char* what) {
        if (count > (buf.size() - off) / sizeof(T)) fail(E8QC_EIO, std::string("short read while loading index (") + what + ")");
        std::vector<T> v(count);
        if (count) std::memcpy(v.data(), take(count * sizeof(T), what), count * sizeof(T));
        return v;
    }
};

// Digits and branch of one block from its rowA byte and (bits-1)-byte field.
void split_decode(int bits, uint8_t rowa, const uint8_t* field, uint32_t d[8], int* branch) {
    if (bits == 1) {
        uint32_t par = 0;
        for (int i = 0; i < 7; ++i) {
            d[i] = (rowa >> (7 - i)) & 1u;
            par ^= d[i];
        }
        d[7] = par & 1u;
        *branch = rowa & 1;
        return;
    }
    const int c = bits - 1;
    uint32_t f[8];
    for (int i = 0; i < 8; ++i) {
        uint32_t v = 0;
        for (int b = 0; b < c; ++b) {
            const int pos = c * i + b;
            v |= static_cast<uint32_t>((field[pos >> 3] >> (pos & 7)) & 1u) << b;
        }
        f[i] = v;
    }
    uint32_t par = 0;
    for (int i = 0; i < 7; ++i) {
        d[i] = f[i] | (static_cast<uint32_t>((rowa >> (7 - i)) & 1u) << c);
        par ^= f[i] & 1u;
    }
    d[7] = ((f[7] >> 1) << 1) | par | (static_cast<uint32_t>(rowa & 1u) << c);
    *branch = static_cast<int>(f[7] & 1u);
}

// OR `width` bits of `v` into the word stream at bit `pos`.
void put_bits(uint32_t* w, size_t pos, int width, uint32_t v) {
    const size_t wi = pos >> 5;
    const int sh = static_cast<int>(pos & 31);
    w[wi] |= v << sh;
    if (sh + width > 32) w[wi + 1] |= v >> (32 - sh);
}

}  // namespace

E8axParts read_e8ax(const char* path, size_t sign_bytes_for_dim(size_t)) {
    if (path == nullptr) fail(E8QC_EINVAL, "null path");
    std::vector<uint8_t> buf;
    {
        std::unique_ptr<std::FILE, int (*)(std::FILE*)> f(std::fopen(path, "rb"), &std::fclose);
        if (!f) fail(E8QC_EIO, std::string("cannot open index file for reading: ") + path);
        if (std::fseek(f.get(), 0, SEEK_END) != 0) fail(E8QC_EIO, "cannot size the index file");
        const long sz = std::ftell(f.get());
        if (sz < 0) fail(E8QC_EIO, "cannot size the index file");
        std::rewind(f.get());
        buf.resize(static_cast<size_t>(sz));
        if (sz > 0 && std::fread(buf.data(), 1, buf.size(), f.get()) != buf.size())
            fail(E8QC_EIO, "short read while loading index");
    }
    Reader r{buf};
    E8axParts p;
    if (r.scalar<uint32_t>("magic") != kE8axMagic) fail(E8QC_EIO, "not an E8Q index file");
    p.n = r.scalar<uint64_t>("header");
    p.dim = r.scalar<uint64_t>("header");
    p.nlist = r.scalar<uint64_t>("header");
    p.bits = static_cast<int>(r.scalar<uint32_t>("header"));
    const uint64_t rot_bytes = r.scalar<uint64_t>("header");
    if (p.bits < 1 || p.bits > 13 || p.nlist == 0 || p.dim == 0 || p.n > 0xFFFFFFFEull)
        fail(E8QC_EIO, "corrupt E8Q index header");
    if (rot_bytes != sign_bytes_for_dim(p.dim)) fail(E8QC_EIO, "rotator payload size mismatch");
    p.pd = (p.dim + 63) / 64 * 64;
    const size_t n = p.n, nlist = p.nlist, pd = p.pd, B = pd / 8;
    p.ids_compact = r.array<uint32_t>(n, "ids");
    p.signs = r.array<uint8_t>(rot_bytes, "rotator");
    p.mean_rot = r.array<float>(pd, "mean");
    p.cen_rot = r.array<float>(nlist * pd, "centroids");
    p.cn2 = r.array<float>(nlist, "centroid norms");
    p.list_begin = r.array<uint64_t>(nlist + 1, "cluster offsets");
    if (p.list_begin[0] != 0 || p.list_begin[nlist] != n) fail(E8QC_EIO, "cluster offsets inconsistent");
    for (size_t c = 0; c < nlist; ++c)
        if (p.list_begin[c + 1] < p.list_begin[c]) fail(E8QC_EIO, "cluster offsets inconsistent");
    const int cbits = p.bits - 1;
    const size_t batch_bytes = (128 + B * 32 + 63) & ~static_cast<size_t>(63);
    const size_t stride = static_cast<size_t>(B) * cbits;  // refine bytes per vector
    const size_t ref_batch = (stride * 32 + 256 + 63) & ~static_cast<size_t>(63);
    const std::vector<uint64_t> arena_begin = r.array<uint64_t>(nlist + 1, "arena offsets");
    uint64_t expect = 0;
    for (size_t c = 0; c < nlist; ++c) {
        if (arena_begin[c] != expect) fail(E8QC_EIO, "arena offsets inconsistent");
        expect += (p.list_begin[c + 1] - p.list_begin[c] + 31) / 32 * batch_bytes;
    }
    if (arena_begin[nlist] != expect) fail(E8QC_EIO, "arena offsets inconsistent");
    const uint8_t* arena = r.take(expect + 64, "arena");
    const std::vector<uint64_t> ref_begin = r.array<uint64_t>(nlist + 1, "refine offsets");
    expect = 0;
    for (size_t c = 0; c < nlist; ++c) {
        if (ref_begin[c] != expect) fail(E8QC_EIO, "refine arena offsets inconsistent");
        expect += (p.list_begin[c + 1] - p.list_begin[c] + 31) / 32 * ref_batch;
    }
    if (ref_begin[nlist] != expect) fail(E8QC_EIO, "refine arena offsets inconsistent");
    const uint8_t* ref_arena = r.take(expect + 64, "refine arena");
    p.prune_alpha = 1.0f;
    if (buf.size() - r.off >= 12 && r.scalar<uint32_t>("trailer") == kOptMagic) {
        const uint32_t lam_bits = r.scalar<uint32_t>("trailer");
        if (r.scalar<uint32_t>("trailer") != kOptMagic) fail(E8QC_EIO, "build-options trailer corrupt");
        float lam = 0.0f;
        std::memcpy(&lam, &lam_bits, 4);
        if (lam > 0.0f && lam == lam) p.prune_alpha = lam;
    }
    // tiles, slots and the repacked code streams
    p.tile_begin.assign(nlist + 1, 0);
    for (size_t c = 0; c < nlist; ++c)
        p.tile_begin[c + 1] =
            p.tile_begin[c] + static_cast<uint32_t>((p.list_begin[c + 1] - p.list_begin[c] + 31) / 32);
    p.ntiles = p.tile_begin[nlist];
    p.nch = code_chunks(static_cast<int>(pd), p.bits);
    const size_t words = static_cast<size_t>(p.nch) * 4;  // per vector, padded to whole chunks
    p.codes.assign(p.ntiles * static_cast<size_t>(p.nch) * 32, uint4{0u, 0u, 0u, 0u});
    p.slot_ids.assign(p.ntiles * 32, 0xFFFFFFFFu);
    p.g1.assign(p.ntiles * 32, 0.0f);
    p.h3.assign(p.ntiles * 32, 0.0f);
    std::vector<uint32_t> w(words + 1);
    for (size_t c = 0; c < nlist; ++c) {
        const size_t cnt = p.list_begin[c + 1] - p.list_begin[c];
        for (size_t v = 0; v < cnt; ++v) {
            const size_t batch = v / 32, lane = v % 32;
            const uint8_t* rowa = arena + arena_begin[c] + batch * batch_bytes + 128;
            const uint8_t* rec = ref_arena + ref_begin[c] + batch * ref_batch;
            const uint8_t* fld = rec + lane * stride;
            std::fill(w.begin(), w.end(), 0u);
            for (size_t b = 0; b < B; ++b) {
                uint32_t d[8];
                int br = 0;
                split_decode(p.bits, rowa[b * 32 + lane], fld + b * cbits, d, &br);
                const size_t base = b * 8 * static_cast<size_t>(p.bits);
                for (int i = 0; i < 7; ++i) put_bits(w.data(), base + i * p.bits, p.bits, d[i]);
                put_bits(w.data(), base + 7 * p.bits, p.bits, (d[7] & ~1u) | static_cast<uint32_t>(br));
            }
            const size_t slot = static_cast<size_t>(p.tile_begin[c]) * 32 + v;
            const size_t tile = slot >> 5, l = slot & 31;
            for (int ch = 0; ch < p.nch; ++ch)
                p.codes[(tile * p.nch + ch) * 32 + l] = uint4{w[4 * ch], w[4 * ch + 1], w[4 * ch + 2], w[4 * ch + 3]};
            std::memcpy(&p.g1[slot], rec + stride * 32 + lane * 4, 4);
            std::memcpy(&p.h3[slot], rec + stride * 32 + 128 + lane * 4, 4);
            p.slot_ids[slot] = p.ids_compact[p.list_begin[c] + v];
        }
    }
    return p;
}

}  // namespace e8qc
