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
// into this library's per-vector bit streams in 32-vector tiles. The scan-bank
// headers (the reference's pruning banks) are kept as read, for saving the
// index again; the device scans score every candidate exactly. write_e8ax is
// the inverse, with the headers either given or computed from the build's
// bank inputs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
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

// The 128-byte scan-bank header of one 32-vector batch from its vectors'
// bank inputs (WriteOrthoBanks, src/index/e8q_build.cpp:31-80): u8 codes of
// base (rounded down), weight (nearest) and perp (rounded up) against the
// batch's range, then the seven scales.
void ortho_banks(const float* base, const float* weight, const float* perp, size_t cnt, uint8_t* hdr) {
    float bmin = 0.0f, bmax = 0.0f, wmin = 0.0f, wmax = 0.0f, pmin = 0.0f, pmax = 0.0f;
    if (cnt > 0) {
        bmin = bmax = base[0];
        wmin = wmax = weight[0];
        pmin = pmax = perp[0];
        for (size_t i = 1; i < cnt; ++i) {
            bmin = std::min(bmin, base[i]);
            bmax = std::max(bmax, base[i]);
            wmin = std::min(wmin, weight[i]);
            wmax = std::max(wmax, weight[i]);
            pmin = std::min(pmin, perp[i]);
            pmax = std::max(pmax, perp[i]);
        }
    }
    const float wamax = std::max(std::abs(wmin), std::abs(wmax));
    const float bsc = bmax > bmin ? (bmax - bmin) / 255.0f : 1.0f;
    const float wsc = wmax > wmin ? (wmax - wmin) / 255.0f : 1.0f;
    const float psc = pmax > pmin ? (pmax - pmin) / 255.0f : 1.0f;
    std::memset(hdr, 0, 128);
    for (size_t i = 0; i < cnt; ++i) {
        hdr[i] = static_cast<uint8_t>(std::clamp<int>(static_cast<int>((base[i] - bmin) / bsc), 0, 255));
        hdr[32 + i] = static_cast<uint8_t>(std::clamp<int>(static_cast<int>(std::lround((weight[i] - wmin) / wsc)), 0, 255));
        hdr[64 + i] = static_cast<uint8_t>(std::clamp<int>(static_cast<int>(std::ceil((perp[i] - pmin) / psc)), 0, 255));
    }
    const float sc[7] = {bmin, bsc, wmin, wsc, pmin, psc, wamax};
    std::memcpy(hdr + 96, sc, sizeof(sc));
}

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
    p.banks.reserve(static_cast<size_t>(expect / batch_bytes) * 128);
    for (size_t c = 0; c < nlist; ++c)
        for (uint64_t off = arena_begin[c]; off < arena_begin[c + 1]; off += batch_bytes)
            p.banks.insert(p.banks.end(), arena + off, arena + off + 128);
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

void write_e8ax(const char* path, const E8axSave& w) {
    if (path == nullptr) fail(E8QC_EINVAL, "null path");
    const size_t n = w.n, nlist = w.nlist, pd = w.pd, B = pd / 8;
    const int bits = w.bits, cb = bits - 1;
    const size_t batch_bytes = (128 + B * 32 + 63) & ~static_cast<size_t>(63);
    const size_t stride = B * static_cast<size_t>(cb);  // refine bytes per vector
    const size_t ref_batch = (stride * 32 + 256 + 63) & ~static_cast<size_t>(63);
    std::vector<uint64_t> arena_begin(nlist + 1, 0), ref_begin(nlist + 1, 0);
    for (size_t c = 0; c < nlist; ++c) {
        const uint64_t batches = (w.list_begin[c + 1] - w.list_begin[c] + 31) / 32;
        arena_begin[c + 1] = arena_begin[c] + batches * batch_bytes;
        ref_begin[c + 1] = ref_begin[c] + batches * ref_batch;
    }
    std::vector<uint8_t> arena(arena_begin[nlist] + 64, 0), ref(ref_begin[nlist] + 64, 0);
    size_t bank = 0;  // batch index in file order (for headers given as read)
    std::vector<float> ob(32), ow(32), op(32);
    for (size_t c = 0; c < nlist; ++c) {
        const uint64_t p0 = w.list_begin[c], cnt = w.list_begin[c + 1] - p0;
        for (uint64_t b = 0; b * 32 < cnt; ++b, ++bank) {
            uint8_t* rec = arena.data() + arena_begin[c] + b * batch_bytes;
            uint8_t* rrec = ref.data() + ref_begin[c] + b * ref_batch;
            const size_t lo = b * 32, hi = std::min<size_t>(cnt, lo + 32);
            if (w.banks) {
                std::memcpy(rec, w.banks + bank * 128, 128);
            } else {
                for (size_t v = lo; v < hi; ++v) {
                    ob[v - lo] = w.ortho[(p0 + v) * 3 + 0];
                    ow[v - lo] = w.ortho[(p0 + v) * 3 + 1];
                    op[v - lo] = w.ortho[(p0 + v) * 3 + 2];
                }
                ortho_banks(ob.data(), ow.data(), op.data(), hi - lo, rec);
            }
            for (size_t v = lo; v < hi; ++v) {
                const size_t lane = v - lo, p = p0 + v;
                for (size_t blk = 0; blk < B; ++blk) {
                    const uint16_t* d = w.digits + (p * B + blk) * 8;
                    const int br = w.branch[p * B + blk] & 1;
                    // rowA (PackCoarseRow, src/index/e8q_scan.cpp:15-27): the top bit
                    // of digit i at bit 7 - i; bit 0 is the branch at b = 1
                    uint8_t row = 0;
                    for (int i = 0; i < 8; ++i) {
                        const int top = (bits == 1 && i == 7) ? br : ((d[i] >> cb) & 1);
                        row = static_cast<uint8_t>(row | (top << (7 - i)));
                    }
                    rec[128 + blk * 32 + lane] = row;
                    if (bits > 1) {
                        // refine field (PackRefineBlock, src/quantization/e8q_codec.cpp:813-839):
                        // low b-1 bits of digits 0..6, of digit 7 with bit 0 = branch
                        uint8_t* f = rrec + lane * stride + blk * static_cast<size_t>(cb);
                        const uint32_t mask = (1u << cb) - 1u;
                        for (int i = 0; i < 8; ++i) {
                            const uint32_t v8 = i < 7 ? (d[i] & mask) : ((d[7] & ~1u & mask) | static_cast<uint32_t>(br));
                            for (int t = 0; t < cb; ++t)
                                if ((v8 >> t) & 1u) {
                                    const size_t pos = static_cast<size_t>(cb) * i + t;
                                    f[pos >> 3] = static_cast<uint8_t>(f[pos >> 3] | (1u << (pos & 7)));
                                }
                        }
                    }
                }
                std::memcpy(rrec + stride * 32 + lane * 4, w.g1 + p, 4);
                std::memcpy(rrec + stride * 32 + 128 + lane * 4, w.h3 + p, 4);
            }
        }
    }
    std::unique_ptr<std::FILE, int (*)(std::FILE*)> f(std::fopen(path, "wb"), &std::fclose);
    if (!f) fail(E8QC_EIO, std::string("cannot open index file for writing: ") + path);
    bool ok = true;
    auto wr = [&](const void* q, size_t bytes) {
        if (bytes != 0 && std::fwrite(q, 1, bytes, f.get()) != bytes) ok = false;
    };
    const uint32_t magic = kE8axMagic;
    const uint64_t n64 = n, dim64 = w.dim, nl64 = nlist, rot64 = w.sign_bytes;
    const int32_t bits32 = bits;
    wr(&magic, 4);
    wr(&n64, 8);
    wr(&dim64, 8);
    wr(&nl64, 8);
    wr(&bits32, 4);
    wr(&rot64, 8);
    wr(w.ids, n * 4);
    wr(w.signs, w.sign_bytes);
    wr(w.mean_rot, pd * 4);
    wr(w.cen_rot, nlist * pd * 4);
    wr(w.cn2, nlist * 4);
    wr(w.list_begin, (nlist + 1) * 8);
    wr(arena_begin.data(), arena_begin.size() * 8);
    wr(arena.data(), arena.size());
    wr(ref_begin.data(), ref_begin.size() * 8);
    wr(ref.data(), ref.size());
    uint32_t lam_bits = 0;
    std::memcpy(&lam_bits, &w.prune_alpha, 4);
    const uint32_t opt = kOptMagic;
    wr(&opt, 4);
    wr(&lam_bits, 4);
    wr(&opt, 4);
    if (!ok || std::fflush(f.get()) != 0) fail(E8QC_EIO, "short write while saving index");
}

}  // namespace e8qc
