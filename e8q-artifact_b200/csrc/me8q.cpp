// ME8Q (mixed-rate E8Q) index: host side of the C ABI (e8qc_me8q_*).
//
// Build (include/e8qlib/index/me8q.hpp:71-84, src/index/me8q_build.cpp:42-311):
// per-dimension variance (given, or on the device), SAQ's DP plan over 64-dim
// blocks (src/quantization/me8q_plan.cpp:47-167) or a manual "L:B,..." plan,
// one FHT-Kac-4 rotator per coded run (seeds stepped by the golden ratio),
// then on the device, per chunk of rows: residual to the list centroid,
// per-run rotation and norms, the E8Q block encoder per run, (coef, h2) fits
// and packing. Search: per-run query rotation, then the grouped exact scan of
// batched.cu (me8q_grouped_search).
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "e8qc.h"
#include "internal.h"
#include "me8q.h"
#include "precision.h"
#include "serve_target.h"
#include "workspace.h"

namespace e8qc {
void set_last_error(const std::string& s);
bool is_device_ptr(const void* p);
std::vector<uint8_t> rotator_signs(size_t dim, uint64_t seed);
}  // namespace e8qc

using namespace e8qc;

namespace {

constexpr size_t kSegDim = 64;
constexpr int kMaxBitsMe8q = 13;
constexpr uint64_t kDefaultRotSeed = 0x5EED1234ULL;  // BuildOptions::rot_seed (me8q.hpp:38)
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

using Plan = std::vector<std::pair<size_t, int>>;

// SAQ's DP: runs of whole 64-dim blocks at 1..max_bits bits (cost sum var /
// 2^b), a trailing dropped run priced at its variance, budget counted in
// units of 64 bits (b*j + 1 per run), at most nblocks/2 runs for avg_bits >=
// 2, and SAQ's acceptance rule (a complete plan replaces the best only when
// 1% cheaper).
Plan allocate(const std::vector<float>& var, size_t pd, float avg_bits, int max_bits, double extra_bits) {
    const size_t nb = pd / kSegDim;
    const double budget = static_cast<double>(avg_bits) * static_cast<double>(pd) + extra_bits + 64.0;
    const size_t units = (budget > 0.0 ? static_cast<size_t>(budget) : 0) / kSegDim;
    const size_t max_segs = avg_bits < 2.0F ? nb : nb / 2;
    std::vector<double> p1(nb + 1, 0.0);
    for (size_t b = 0; b < nb; ++b) {
        double s = 0.0;
        for (size_t k = 0; k < kSegDim; ++k) s += static_cast<double>(var[b * kSegDim + k]);
        p1[b + 1] = p1[b] + s;
    }
    const size_t si = nb + 1, st = units + 1;
    std::vector<double> f((max_segs + 1) * si * st, DBL_MAX);
    std::vector<uint32_t> pred(f.size(), 0);
    auto at = [&](size_t ns, size_t i, size_t t) { return (ns * si + i) * st + t; };
    f[at(0, 0, 0)] = 0.0;
    double best = DBL_MAX;
    size_t ans_ns = 0, ans_t = 0;
    for (size_t ns = 0; ns <= max_segs; ++ns)
        for (size_t i = 0; i <= nb; ++i)
            for (size_t t = 0; t <= units; ++t) {
                const double cur = f[at(ns, i, t)];
                if (cur >= DBL_MAX) continue;
                if (i == nb) {
                    if (cur * 1.01 < best) {
                        best = cur;
                        ans_ns = ns;
                        ans_t = t;
                    }
                    continue;
                }
                if (ns == max_segs) continue;
                for (size_t j = 1; i + j <= nb; ++j) {
                    const double vsum = p1[i + j] - p1[i];
                    for (int b = 1; b <= max_bits; ++b) {
                        const size_t t2 = t + static_cast<size_t>(b) * j + 1;
                        if (t2 > units) break;
                        const double v = cur + vsum / static_cast<double>(int64_t{1} << b);
                        const size_t to = at(ns + 1, i + j, t2);
                        if (v < f[to]) {
                            f[to] = v;
                            pred[to] = static_cast<uint32_t>((i << 4) | static_cast<size_t>(b));
                        }
                    }
                }
                const double rest = p1[nb] - p1[i];
                const size_t to = at(ns + 1, nb, t);
                if (cur + rest < f[to]) {
                    f[to] = cur + rest;
                    pred[to] = static_cast<uint32_t>(i << 4);
                }
            }
    if (best >= DBL_MAX) return Plan{{pd, 0}};  // no feasible plan: everything dropped
    Plan plan;
    size_t ns = ans_ns, i = nb, t = ans_t;
    while (i > 0) {
        const uint32_t p = pred[at(ns, i, t)];
        const size_t prev = p >> 4;
        const int b = static_cast<int>(p & 0xFu);
        plan.push_back({(i - prev) * kSegDim, b});
        --ns;
        if (b != 0) t -= static_cast<size_t>(b) * (i - prev) + 1;
        i = prev;
    }
    std::reverse(plan.begin(), plan.end());
    return plan;
}

// "L:B,L:B,..." (src/index/me8q_common.cpp:37-68): empty tokens skipped,
// numbers read like atol, L a positive multiple of 64, B in [0, 13], the
// runs covering the padded dimension exactly.
Plan parse_plan(const std::string& spec, size_t pd) {
    Plan plan;
    size_t total = 0;
    std::string tok;
    auto take = [&] {
        if (tok.empty()) return;
        const size_t colon = tok.find(':');
        if (colon == std::string::npos) fail(E8QC_EINVAL, "plan_spec: expected L:B, got " + tok);
        const long len = std::strtol(tok.c_str(), nullptr, 10);
        const long bits = std::strtol(tok.c_str() + colon + 1, nullptr, 10);
        if (len <= 0 || len % static_cast<long>(kSegDim) != 0 || bits < 0 || bits > kMaxBitsMe8q)
            fail(E8QC_EINVAL, "plan_spec: bad run " + tok);
        plan.emplace_back(static_cast<size_t>(len), static_cast<int>(bits));
        total += static_cast<size_t>(len);
        tok.clear();
    };
    for (const char ch : spec) {
        if (ch == ',') take();
        else tok.push_back(ch);
    }
    take();
    if (total != pd)
        fail(E8QC_EINVAL, "plan_spec: runs cover " + std::to_string(total) + " of " + std::to_string(pd) +
                              " padded dims");
    return plan;
}

struct DeviceGuard {
    int prev = 0;
    explicit DeviceGuard(int d) {
        E8QC_CUDA(cudaGetDevice(&prev));
        E8QC_CUDA(cudaSetDevice(d));
    }
    ~DeviceGuard() { cudaSetDevice(prev); }
};

int guarded(const std::function<void()>& f) {
    try {
        f();
        return E8QC_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return E8QC_ENOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return E8QC_EINVAL;
    }
}

}  // namespace

struct e8qc_me8q {
    int device = 0;
    size_t dim = 0, pd = 0;
    float avg_bits = 4.0F;
    uint64_t seed = 0;
    // what an ME8QIDXX file records besides the data (Me8qIndex::Save)
    uint64_t rot_seed = 0;   // the effective rotator seed of the plan's runs
    int max_bits = 13;
    bool drop_energy = true;
    float prune_alpha = 0.0F;
    std::vector<uint8_t> signs_host;  // the coded runs' rotator signs, in plan order
    bool built = false;
    size_t n = 0, nlist = 0, ntiles = 0, nslots = 0;
    int nch = 0, ncoded = 0, route_dim = 0;
    size_t bytes_per_vector = 0;
    Plan plan;
    std::vector<Me8qRun> runs;
    std::vector<Me8qChunk> chunks;
    std::vector<uint64_t> list_begin;
    std::vector<uint32_t> tile_begin, ids_compact, inv_pos;
    std::vector<float> cen_host;  // padded centroids (estimate)
    DevBuf runs_d, chunks_d, levels, signs, cen_pad, cen_rot, cn2, tile_begin_d, list_len_d, list_order_d,
        list_of_tile_d, ids, codes, coef, h2, hsum, list_begin_d;
    DevBuf proxy, sigma;                 // precision mode: int8 proxy plane and per-slot scale (built on first use)
    // pruned mode: the fast layout (me8q_fast.cu), built on first use
    DevBuf f_runs, f_plane, f_gain, f_vpc, f_bank, f_scl, f_rcn2;
    Me8qFast fast{};
    std::vector<uint64_t> tiles_prefix;  // prefix sums of the lists' tile counts, largest first
    Me8qView view{};
    Workspace ws;
    std::mutex mu;
    std::map<uint64_t, std::pair<int, int>> tuned;  // (schedule, stages) per (mode, log2 nq, log2 nprobe)
    std::mutex tune_mu;
    size_t memory_bytes() const {
        return runs_d.bytes + chunks_d.bytes + levels.bytes + signs.bytes + cen_pad.bytes + cen_rot.bytes + cn2.bytes +
               tile_begin_d.bytes + list_len_d.bytes + list_order_d.bytes + list_of_tile_d.bytes + ids.bytes +
               codes.bytes + coef.bytes + h2.bytes + hsum.bytes + list_begin_d.bytes + proxy.bytes + sigma.bytes +
               f_runs.bytes + f_plane.bytes + f_gain.bytes + f_vpc.bytes + f_bank.bytes + f_scl.bytes + f_rcn2.bytes;
    }
};

namespace {

void require_built(const e8qc_me8q* x, const char* what) {
    if (x == nullptr) fail(E8QC_EINVAL, "null index");
    if (!x->built) fail(E8QC_ESTATE, std::string("Me8qIndex must be built or loaded before ") + what);
}

// Plan -> run descriptors, rotator signs, chunk table and level tables.
void layout_plan(e8qc_me8q* x, uint64_t rot_seed, cudaStream_t s) {
    x->runs.clear();
    x->chunks.clear();
    std::vector<uint8_t> sg_all;
    std::vector<float> lev_all;
    int lev_off[kMaxBitsMe8q + 1];
    std::fill(lev_off, lev_off + kMaxBitsMe8q + 1, -1);
    uint64_t sd = rot_seed;
    size_t off = 0, word = 0;
    int coded = 0;
    for (const auto& seg : x->plan) {
        Me8qRun r{};
        r.off = static_cast<int>(off);
        r.len = static_cast<int>(seg.first);
        r.bits = seg.second;
        r.coded = seg.second != 0 ? coded : -1;
        int td = 1;
        while ((td << 1) <= r.len) td <<= 1;
        r.td = td;
        r.fac = 1.0f / std::sqrt(static_cast<float>(td));
        r.soff = static_cast<int>(sg_all.size());
        r.word0 = static_cast<int>(word);
        if (seg.second != 0) {
            sd += kGolden;  // BuildRunRotators (me8q_build.cpp:29-40)
            const std::vector<uint8_t> sg = rotator_signs(seg.first, sd);
            sg_all.insert(sg_all.end(), sg.begin(), sg.end());
            if (lev_off[seg.second] < 0) {
                lev_off[seg.second] = static_cast<int>(lev_all.size());
                for (int br = 0; br < 2; ++br) {
                    const std::vector<double> lv = branch_levels(seg.second, br);
                    for (double d : lv) lev_all.push_back(static_cast<float>(d));
                }
            }
            word += seg.first * static_cast<size_t>(seg.second) / 32;
            ++coded;
        }
        x->runs.push_back(r);
        off += seg.first;
    }
    x->ncoded = coded;
    x->route_dim = static_cast<int>(x->pd);
    for (auto it = x->plan.rbegin(); it != x->plan.rend() && it->second == 0; ++it)
        x->route_dim -= static_cast<int>(it->first);
    for (const auto& r : x->runs) {
        if (r.off >= x->route_dim) break;
        for (int c = 0; c < r.len / 64; ++c)
            x->chunks.push_back(Me8qChunk{r.bits, r.coded, r.word0 + c * 2 * r.bits, r.bits ? lev_off[r.bits] : 0});
    }
    const size_t stream_bits = word * 32;
    x->nch = static_cast<int>(std::max<size_t>(1, (stream_bits + 127) / 128));
    x->bytes_per_vector = static_cast<size_t>(coded) * 8;
    for (const auto& seg : x->plan)
        if (seg.second) x->bytes_per_vector += seg.first / 8 * static_cast<size_t>(seg.second);
    x->rot_seed = rot_seed;
    x->signs_host = sg_all;
    if (lev_all.empty()) lev_all.push_back(0.0f);
    if (sg_all.empty()) sg_all.push_back(0);
    x->runs_d.upload(x->runs.data(), x->runs.size() * sizeof(Me8qRun), s);
    std::vector<Me8qChunk> chunk_tab = x->chunks;
    if (chunk_tab.empty()) chunk_tab.push_back(Me8qChunk{0, -1, 0, 0});  // all runs dropped
    x->chunks_d.upload(chunk_tab.data(), chunk_tab.size() * sizeof(Me8qChunk), s);
    x->levels.upload(lev_all.data(), lev_all.size() * 4, s);
    x->signs.upload(sg_all.data(), sg_all.size(), s);
}

void fill_view(e8qc_me8q* x) {
    Me8qView& v = x->view;
    v = Me8qView{};
    DevIndex& b = v.base;
    b.dim = static_cast<int>(x->dim);
    b.pd = static_cast<int>(x->pd);
    b.B = static_cast<int>(x->pd / 8);
    b.bits = 0;
    b.nlist = static_cast<int>(x->nlist);
    b.nch = x->nch;
    b.ntiles = static_cast<int>(x->ntiles);
    b.cen = x->cen_rot.as<float>();
    b.cn2 = x->cn2.as<float>();
    b.tile_begin = x->tile_begin_d.as<uint32_t>();
    b.list_len = x->list_len_d.as<uint32_t>();
    b.codes = static_cast<const uint4*>(x->codes.p);
    b.ids = x->ids.as<uint32_t>();
    b.list_order = x->list_order_d.as<uint32_t>();
    b.list_of_tile = x->list_of_tile_d.as<uint32_t>();
    b.h3 = x->hsum.as<float>();       // precision scan epilogue: (d2 + hsum) - 2 sigma S'
    b.g1 = x->sigma.as<const float>();
    b.proxy = static_cast<const uint4*>(x->proxy.p);
    v.coef = x->coef.as<float>();
    v.h2 = x->h2.as<float>();
    v.hsum = x->hsum.as<float>();
    v.runs = x->runs_d.as<Me8qRun>();
    v.chunks = x->chunks_d.as<Me8qChunk>();
    v.levels = x->levels.as<float>();
    v.signs = x->signs.as<uint8_t>();
    v.nruns = static_cast<int>(x->runs.size());
    v.ncoded = x->ncoded;
    v.nchunks = static_cast<int>(x->chunks.size());
    v.route_dim = x->route_dim;
    v.nslots = x->nslots;
}

// Lists of cnt[c] vectors in 32-vector tiles: offsets, tiles, work-queue
// orders (longest first, then list id), the tile -> list map; uploads them.
// A new layout drops the precision plane.
void setup_lists(e8qc_me8q* x, const std::vector<uint32_t>& cnt, cudaStream_t s) {
    const size_t nlist = x->nlist;
    x->list_begin.assign(nlist + 1, 0);
    x->tile_begin.assign(nlist + 1, 0);
    for (size_t c = 0; c < nlist; ++c) {
        x->list_begin[c + 1] = x->list_begin[c] + cnt[c];
        x->tile_begin[c + 1] = x->tile_begin[c] + (cnt[c] + 31) / 32;
    }
    x->ntiles = x->tile_begin[nlist];
    x->nslots = x->ntiles * 32;
    x->proxy.release();
    x->sigma.release();
    x->f_plane.release();
    x->fast = Me8qFast{};
    {
        std::vector<uint64_t> t(nlist);
        for (size_t c = 0; c < nlist; ++c) t[c] = x->tile_begin[c + 1] - x->tile_begin[c];
        std::sort(t.rbegin(), t.rend());
        x->tiles_prefix.assign(nlist + 1, 0);
        for (size_t c = 0; c < nlist; ++c) x->tiles_prefix[c + 1] = x->tiles_prefix[c] + t[c];
    }
    std::vector<uint32_t> list_len(nlist), list_of_tile(std::max<size_t>(1, x->ntiles), 0), order(2 * nlist);
    for (size_t c = 0; c < nlist; ++c) {
        list_len[c] = cnt[c];
        for (uint32_t t = x->tile_begin[c]; t < x->tile_begin[c + 1]; ++t) list_of_tile[t] = static_cast<uint32_t>(c);
        order[c] = order[nlist + c] = static_cast<uint32_t>(c);
    }
    std::stable_sort(order.begin(), order.begin() + nlist, [&](uint32_t a, uint32_t b) { return cnt[a] > cnt[b]; });
    x->tile_begin_d.upload(x->tile_begin.data(), x->tile_begin.size() * 4, s);
    x->list_len_d.upload(list_len.data(), nlist * 4, s);
    x->list_order_d.upload(order.data(), order.size() * 4, s);
    x->list_of_tile_d.upload(list_of_tile.data(), list_of_tile.size() * 4, s);
    x->list_begin_d.upload(x->list_begin.data(), x->list_begin.size() * 8, s);
}

// Zeroed code / factor storage for the layout, and the centroids: padded
// (nlist x pd) -> per-run rotated on the device -> ||.||^2 in fp64 on the host
// (include/e8qlib/index/ivf_common.hpp:43-54). Leaves the view filled.
void setup_storage(e8qc_me8q* x, std::vector<float> cen_padded, cudaStream_t s) {
    const size_t nlist = x->nlist, pd = x->pd;
    x->cen_host = std::move(cen_padded);
    x->cen_pad.upload(x->cen_host.data(), x->cen_host.size() * 4, s);
    x->cen_rot.alloc(nlist * pd * 4);
    x->codes.alloc(std::max<size_t>(1, x->ntiles) * x->nch * 32 * 16);
    E8QC_CUDA(cudaMemsetAsync(x->codes.p, 0, x->codes.bytes, s));
    const size_t nc = std::max(1, x->ncoded);
    x->coef.alloc(nc * std::max<size_t>(1, x->nslots) * 4);
    x->h2.alloc(nc * std::max<size_t>(1, x->nslots) * 4);
    x->hsum.alloc(std::max<size_t>(1, x->nslots) * 4);
    E8QC_CUDA(cudaMemsetAsync(x->coef.p, 0, x->coef.bytes, s));
    E8QC_CUDA(cudaMemsetAsync(x->h2.p, 0, x->h2.bytes, s));
    x->cn2.alloc(nlist * 4);
    fill_view(x);
    launch_me8q_prep(x->cen_pad.as<float>(), pd, static_cast<int>(pd), static_cast<int>(pd), nullptr, nullptr, x->view,
                     0, nlist, x->cen_rot.as<float>(), nullptr, nullptr, s);
    std::vector<float> cr(nlist * pd), n2(nlist);
    E8QC_CUDA(cudaMemcpyAsync(cr.data(), x->cen_rot.p, cr.size() * 4, cudaMemcpyDeviceToHost, s));
    E8QC_CUDA(cudaStreamSynchronize(s));
    for (size_t c = 0; c < nlist; ++c) {
        double acc = 0.0;
        for (size_t d = 0; d < pd; ++d)
            acc = std::fma(static_cast<double>(cr[c * pd + d]), static_cast<double>(cr[c * pd + d]), acc);
        n2[c] = static_cast<float>(acc);
    }
    E8QC_CUDA(cudaMemcpyAsync(x->cn2.p, n2.data(), nlist * 4, cudaMemcpyHostToDevice, s));
    E8QC_CUDA(cudaStreamSynchronize(s));
}

void build(e8qc_me8q* x, const float* data, size_t n, const float* centroids, size_t nlist, const uint32_t* cluster_ids,
           const e8qc_me8q_build_opts* o, cudaStream_t s) {
    const size_t dim = x->dim, pd = x->pd;
    DevBuf tdata;
    const float* xd = data;
    if (!is_device_ptr(data)) {
        tdata.alloc(n * dim * 4);
        E8QC_CUDA(cudaMemcpyAsync(tdata.p, data, n * dim * 4, cudaMemcpyHostToDevice, s));
        xd = tdata.as<float>();
    }
    std::vector<float> cen(nlist * dim);
    if (is_device_ptr(centroids)) E8QC_CUDA(cudaMemcpy(cen.data(), centroids, cen.size() * 4, cudaMemcpyDeviceToHost));
    else std::memcpy(cen.data(), centroids, cen.size() * 4);
    std::vector<uint32_t> cid(n);
    if (is_device_ptr(cluster_ids)) E8QC_CUDA(cudaMemcpy(cid.data(), cluster_ids, n * 4, cudaMemcpyDeviceToHost));
    else std::memcpy(cid.data(), cluster_ids, n * 4);
    for (size_t i = 0; i < n; ++i)
        if (cid[i] >= nlist) fail(E8QC_EINVAL, "cluster_ids out of range");
    // ---- plan ----
    const int max_bits = (o && o->max_bits > 0) ? o->max_bits : kMaxBitsMe8q;
    if (max_bits < 1 || max_bits > kMaxBitsMe8q) fail(E8QC_EINVAL, "max_bits must be in [1, 13]");
    if (o && o->plan_spec && o->plan_spec[0]) {
        x->plan = parse_plan(o->plan_spec, pd);
    } else {
        std::vector<float> var(pd, 0.0f);
        if (o && o->variance) {
            if (is_device_ptr(o->variance)) E8QC_CUDA(cudaMemcpy(var.data(), o->variance, dim * 4, cudaMemcpyDeviceToHost));
            else std::memcpy(var.data(), o->variance, dim * 4);
        } else {
            DevBuf vd;
            vd.alloc(dim * 4);
            launch_me8q_variance(xd, n, static_cast<int>(dim), vd.as<float>(), s);
            E8QC_CUDA(cudaMemcpyAsync(var.data(), vd.p, dim * 4, cudaMemcpyDeviceToHost, s));
            E8QC_CUDA(cudaStreamSynchronize(s));
        }
        x->plan = allocate(var, pd, x->avg_bits, max_bits, o ? o->extra_budget_bits : 0.0);
    }
    if (x->plan.size() > 256) fail(E8QC_EINVAL, "a plan may have at most 256 runs");
    const uint64_t rot_seed = x->seed != 0 ? x->seed : kDefaultRotSeed;
    layout_plan(x, rot_seed, s);
    // ---- lists: tiles of 32 slots, rows in file order within a list ----
    x->n = n;
    x->nlist = nlist;
    std::vector<uint32_t> cnt(nlist, 0);
    for (size_t i = 0; i < n; ++i) ++cnt[cid[i]];
    setup_lists(x, cnt, s);
    std::vector<uint32_t> slot_of_row(n), slot_ids(std::max<size_t>(1, x->nslots), 0xFFFFFFFFu), fillc(nlist, 0);
    x->ids_compact.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
        const uint32_t c = cid[i];
        const uint32_t local = fillc[c]++;
        slot_of_row[i] = x->tile_begin[c] * 32 + local;
        slot_ids[slot_of_row[i]] = static_cast<uint32_t>(i);
        x->ids_compact[x->list_begin[c] + local] = static_cast<uint32_t>(i);
    }
    x->inv_pos.clear();
    x->ids.upload(slot_ids.data(), slot_ids.size() * 4, s);
    {
        std::vector<float> padded(nlist * pd, 0.0f);
        for (size_t c = 0; c < nlist; ++c) std::memcpy(&padded[c * pd], &cen[c * dim], dim * 4);
        setup_storage(x, std::move(padded), s);
    }
    const size_t nc = std::max(1, x->ncoded);
    // ---- encode in chunks of rows ----
    DevBuf cid_d, slot_d, rr, norm2, drop, dg, br;
    cid_d.upload(cid.data(), n * 4, s);
    slot_d.upload(slot_of_row.data(), n * 4, s);
    const size_t chunk = std::min<size_t>(n, 1u << 18);
    rr.alloc(chunk * pd * 4);
    norm2.alloc(chunk * nc * 8);
    drop.alloc(chunk * 8);
    dg.alloc(chunk * pd * 2);
    br.alloc(chunk * (pd / 8));
    const int dev = x->device;
    const bool drop_energy = o ? o->drop_energy != 0 : true;
    x->max_bits = max_bits;
    x->drop_energy = drop_energy;
    x->prune_alpha = o ? o->prune_alpha : 0.0F;
    for (size_t r0 = 0; r0 < n; r0 += chunk) {
        const size_t m = std::min(chunk, n - r0);
        launch_me8q_prep(xd, dim, static_cast<int>(dim), static_cast<int>(pd), x->cen_pad.as<float>(),
                         cid_d.as<uint32_t>(), x->view, r0, m, rr.as<float>(), norm2.as<double>(), drop.as<double>(), s);
        for (const auto& run : x->runs) {
            if (run.bits == 0) continue;
            const double srd = fixed_scale(run.bits) * std::sqrt(static_cast<double>(run.len));
            launch_me8q_encode(enc_tables_device(dev, run.bits), rr.as<float>(), static_cast<int>(pd), norm2.as<double>(),
                               x->ncoded, run.coded, run.off, run.len, m, srd, dg.as<uint16_t>(), br.as<uint8_t>(), s);
        }
        launch_me8q_fits_pack(x->view, rr.as<float>(), dg.as<uint16_t>(), br.as<uint8_t>(), norm2.as<double>(),
                              drop.as<double>(), cid_d.as<uint32_t>(), x->cen_rot.as<float>(), static_cast<int>(pd), r0, m,
                              slot_d.as<uint32_t>(), drop_energy, static_cast<uint4*>(x->codes.p), x->coef.as<float>(),
                              x->h2.as<float>(), s);
    }
    launch_me8q_hsum(x->view, x->hsum.as<float>(), s);
    E8QC_CUDA(cudaStreamSynchronize(s));
    x->built = true;
}

// Reader of the reference's ME8Q index file (ME8QIDXX; Me8qIndex::Save /
// Load, src/index/me8q_io.cpp:29-175): header (n, dim, padded dim, lists,
// bytes per vector), avg_bits and the option flags, the plan, the padded
// centroids, cluster-major ids, list and byte offsets, the rows, the rotator
// seed and each coded run's rotator signs. A row is the (coef, h2) pair of
// every coded run, then the runs' blocks of b bytes each: digits 0..6 at b
// bits, digit 7 without its parity bit at b - 1 bits, the branch in the top
// bit (src/quantization/me8q_codec.cpp:109-129). The rows are unpacked and
// repacked into this library's streams; nothing is re-encoded.
void load_me8q_file(e8qc_me8q* x, const char* path, cudaStream_t s) {
    if (path == nullptr) fail(E8QC_EINVAL, "null path");
    std::vector<uint8_t> buf;
    {
        std::unique_ptr<std::FILE, int (*)(std::FILE*)> f(std::fopen(path, "rb"), &std::fclose);
        if (!f) fail(E8QC_EIO, std::string("Me8qIndex::Load: cannot read ") + path);
        if (std::fseek(f.get(), 0, SEEK_END) != 0) fail(E8QC_EIO, "cannot size the index file");
        const long sz = std::ftell(f.get());
        if (sz < 0) fail(E8QC_EIO, "cannot size the index file");
        std::rewind(f.get());
        buf.resize(static_cast<size_t>(sz));
        if (sz > 0 && std::fread(buf.data(), 1, buf.size(), f.get()) != buf.size())
            fail(E8QC_EIO, "short read while loading index");
    }
    size_t off = 0;
    auto take = [&](size_t bytes, const char* what) {
        if (bytes > buf.size() - off) fail(E8QC_EIO, std::string("Me8qIndex::Load: short read (") + what + ")");
        const uint8_t* p = buf.data() + off;
        off += bytes;
        return p;
    };
    auto u64 = [&](const char* what) {
        uint64_t v;
        std::memcpy(&v, take(8, what), 8);
        return v;
    };
    if (std::memcmp(take(8, "magic"), "ME8QIDXX", 8) != 0) fail(E8QC_EIO, std::string("Me8qIndex::Load: bad magic ") + path);
    const uint64_t n = u64("header"), dim = u64("header"), pd = u64("header"), nlist = u64("header");
    u64("header");  // bytes per vector: recomputed from the plan
    float avg = 0.0f;
    std::memcpy(&avg, take(4, "avg_bits"), 4);
    int32_t flags[4];
    std::memcpy(flags, take(16, "flags"), 16);
    if (dim == 0 || dim > 16384 || pd != (dim + 63) / 64 * 64 || nlist == 0 || n > 0xFFFFFFFEull)
        fail(E8QC_EIO, "Me8qIndex::Load: corrupt header");
    if (dim != x->dim) fail(E8QC_EINVAL, "index file dimension does not match the index");
    const uint64_t nplan = u64("plan");
    if (nplan == 0 || nplan > 256) fail(E8QC_EIO, "Me8qIndex::Load: corrupt plan");
    Plan plan;
    size_t covered = 0;
    for (uint64_t i = 0; i < nplan; ++i) {
        const uint64_t len = u64("plan");
        int32_t bits = 0;
        std::memcpy(&bits, take(4, "plan"), 4);
        if (len == 0 || len % kSegDim != 0 || bits < 0 || bits > kMaxBitsMe8q) fail(E8QC_EIO, "Me8qIndex::Load: corrupt plan");
        plan.emplace_back(static_cast<size_t>(len), bits);
        covered += static_cast<size_t>(len);
    }
    if (covered != pd) fail(E8QC_EIO, "Me8qIndex::Load: plan does not cover the padded dimension");
    if (nlist > (buf.size() - off) / (pd * 4)) fail(E8QC_EIO, "Me8qIndex::Load: short read (centroids)");
    std::vector<float> cen(nlist * pd);
    std::memcpy(cen.data(), take(cen.size() * 4, "centroids"), cen.size() * 4);
    if (n > (buf.size() - off) / 4) fail(E8QC_EIO, "Me8qIndex::Load: short read (ids)");
    std::vector<uint32_t> ids(n);
    if (n) std::memcpy(ids.data(), take(n * 4, "ids"), n * 4);
    std::vector<uint64_t> lb(nlist + 1), bb(nlist + 1);
    std::memcpy(lb.data(), take(lb.size() * 8, "list_begin"), lb.size() * 8);
    std::memcpy(bb.data(), take(bb.size() * 8, "byte_begin"), bb.size() * 8);
    // per-row stride from the plan (coef, h2 per coded run + b bytes per block)
    size_t nseg = 0, stride = 0;
    for (const auto& seg : plan)
        if (seg.second) {
            ++nseg;
            stride += seg.first / 8 * static_cast<size_t>(seg.second);
        }
    stride += nseg * 8;
    if (lb[0] != 0 || lb[nlist] != n || bb[0] != 0) fail(E8QC_EIO, "Me8qIndex::Load: offsets inconsistent");
    for (uint64_t c = 0; c < nlist; ++c)
        if (lb[c + 1] < lb[c] || bb[c + 1] - bb[c] != (lb[c + 1] - lb[c]) * stride)
            fail(E8QC_EIO, "Me8qIndex::Load: offsets inconsistent");
    const uint8_t* rows = take(bb[nlist], "codes");
    const uint64_t rot_seed = u64("rot_seed");
    const uint64_t n_rot = u64("rotator count");
    if (n_rot != nseg) fail(E8QC_EIO, "Me8qIndex::Load: rotator count mismatch");
    std::vector<uint8_t> file_signs;
    for (uint64_t r = 0; r < n_rot; ++r) {
        const uint64_t bytes = u64("rot_bytes");
        const uint8_t* p = take(bytes, "rotator");
        file_signs.insert(file_signs.end(), p, p + bytes);
    }
    // index state: plan, runs and rotators (the file's signs), lists, storage
    x->avg_bits = avg;
    x->seed = rot_seed;
    x->max_bits = flags[1];
    x->drop_energy = flags[2] != 0;
    std::memcpy(&x->prune_alpha, &flags[3], 4);
    x->plan = plan;
    layout_plan(x, rot_seed, s);
    {
        size_t want = 0;
        for (const auto& run : x->runs)
            if (run.bits) want += rotator_signs(static_cast<size_t>(run.len), 0).size();
        if (want != file_signs.size()) fail(E8QC_EIO, "Me8qIndex::Load: rotator payload size mismatch");
        if (!file_signs.empty()) x->signs.upload(file_signs.data(), file_signs.size(), s);
        x->signs_host = file_signs;
    }
    x->n = n;
    x->nlist = nlist;
    std::vector<uint32_t> cnt(nlist);
    for (uint64_t c = 0; c < nlist; ++c) cnt[c] = static_cast<uint32_t>(lb[c + 1] - lb[c]);
    setup_lists(x, cnt, s);
    std::vector<uint32_t> slot_ids(std::max<size_t>(1, x->nslots), 0xFFFFFFFFu);
    for (uint64_t c = 0; c < nlist; ++c)
        for (uint64_t r = lb[c]; r < lb[c + 1]; ++r) slot_ids[x->tile_begin[c] * 32 + (r - lb[c])] = ids[r];
    x->ids_compact = ids;
    x->inv_pos.clear();
    x->ids.upload(slot_ids.data(), slot_ids.size() * 4, s);
    setup_storage(x, std::move(cen), s);
    // rows -> streams and factor planes
    const size_t nc = static_cast<size_t>(std::max(1, x->ncoded));
    std::vector<uint4> codes(std::max<size_t>(1, x->ntiles) * x->nch * 32, uint4{0u, 0u, 0u, 0u});
    std::vector<float> coef(nc * std::max<size_t>(1, x->nslots), 0.0f), h2(coef.size(), 0.0f);
    std::vector<uint32_t> w(static_cast<size_t>(x->nch) * 4 + 1);
    for (uint64_t c = 0; c < nlist; ++c)
        for (uint64_t r = 0; r < lb[c + 1] - lb[c]; ++r) {
            const uint8_t* row = rows + bb[c] + r * stride;
            const size_t slot = static_cast<size_t>(x->tile_begin[c]) * 32 + r;
            for (size_t q = 0; q < nseg; ++q) {
                std::memcpy(&coef[q * x->nslots + slot], row + 8 * q, 4);
                std::memcpy(&h2[q * x->nslots + slot], row + 8 * q + 4, 4);
            }
            std::fill(w.begin(), w.end(), 0u);
            const uint8_t* cur = row + nseg * 8;
            for (const auto& run : x->runs) {
                if (run.bits == 0) continue;
                const int b = run.bits;
                for (int blk = 0; blk < run.len / 8; ++blk, cur += b) {
                    auto bit_at = [&](int pos) { return static_cast<uint32_t>((cur[pos >> 3] >> (pos & 7)) & 1u); };
                    auto get = [&](int pos, int width) {
                        uint32_t v = 0;
                        for (int t = 0; t < width; ++t) v |= bit_at(pos + t) << t;
                        return v;
                    };
                    const size_t base = static_cast<size_t>(run.word0) * 32 + static_cast<size_t>(blk) * 8 * b;
                    for (int i = 0; i < 7; ++i) {
                        const uint32_t d = get(b * i, b);
                        const size_t pos = base + static_cast<size_t>(i) * b;
                        w[pos >> 5] |= d << (pos & 31);
                        if ((pos & 31) + b > 32) w[(pos >> 5) + 1] |= d >> (32 - (pos & 31));
                    }
                    // digit 7 field: its bits 1..b-1 and the branch in bit 0
                    const uint32_t f7 = (get(b * 7, b - 1) << 1) | bit_at(8 * b - 1);
                    const size_t pos = base + static_cast<size_t>(7) * b;
                    w[pos >> 5] |= f7 << (pos & 31);
                    if ((pos & 31) + b > 32) w[(pos >> 5) + 1] |= f7 >> (32 - (pos & 31));
                }
            }
            const size_t tile = slot >> 5, l = slot & 31;
            for (int ch = 0; ch < x->nch; ++ch)
                codes[(tile * x->nch + ch) * 32 + l] = uint4{w[4 * ch], w[4 * ch + 1], w[4 * ch + 2], w[4 * ch + 3]};
        }
    E8QC_CUDA(cudaMemcpyAsync(x->codes.p, codes.data(), codes.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
    if (x->ncoded > 0) {
        E8QC_CUDA(cudaMemcpyAsync(x->coef.p, coef.data(), coef.size() * 4, cudaMemcpyHostToDevice, s));
        E8QC_CUDA(cudaMemcpyAsync(x->h2.p, h2.data(), h2.size() * 4, cudaMemcpyHostToDevice, s));
    }
    launch_me8q_hsum(x->view, x->hsum.as<float>(), s);
    E8QC_CUDA(cudaStreamSynchronize(s));
    x->built = true;
}

// Writer of the reference's ME8QIDXX layout (Me8qIndex::Save,
// src/index/me8q_io.cpp:29-65), from the device index: digits and branch of
// every slot come back through the decode kernel, (coef, h2) from the factor
// planes, and each row is packed as the reference packs it (PackSegment /
// PackBlock, src/quantization/me8q_codec.cpp:109-151: per block of a coded
// run, digits 0..6 at b bits, digit 7 without its parity bit at b - 1 bits,
// the branch in the block's top bit). The reference loads such a file.
void save_me8q_file(e8qc_me8q* x, const char* path, cudaStream_t s) {
    if (path == nullptr) fail(E8QC_EINVAL, "null path");
    const size_t n = x->n, pd = x->pd, nlist = x->nlist, B = pd / 8;
    std::vector<uint16_t> dg(n * pd);
    std::vector<uint8_t> br(n * B);
    {
        DevBuf dd, bb;
        dd.alloc(std::max<size_t>(1, n * pd * 2));
        bb.alloc(std::max<size_t>(1, n * B));
        launch_me8q_decode(x->view, static_cast<int>(x->ntiles), x->list_of_tile_d.as<uint32_t>(),
                           x->list_begin_d.as<uint64_t>(), static_cast<int>(pd), dd.as<uint16_t>(), bb.as<uint8_t>(), s);
        E8QC_CUDA(cudaMemcpyAsync(dg.data(), dd.p, n * pd * 2, cudaMemcpyDeviceToHost, s));
        E8QC_CUDA(cudaMemcpyAsync(br.data(), bb.p, n * B, cudaMemcpyDeviceToHost, s));
        E8QC_CUDA(cudaStreamSynchronize(s));
    }
    const size_t nc = static_cast<size_t>(x->ncoded);
    std::vector<float> cf(nc * x->nslots), hh(nc * x->nslots);
    if (nc) {
        E8QC_CUDA(cudaMemcpy(cf.data(), x->coef.p, cf.size() * 4, cudaMemcpyDeviceToHost));
        E8QC_CUDA(cudaMemcpy(hh.data(), x->h2.p, hh.size() * 4, cudaMemcpyDeviceToHost));
    }
    const size_t stride = x->bytes_per_vector;
    std::vector<uint8_t> rows(n * stride, 0);
    for (size_t c = 0; c < nlist; ++c)
        for (uint64_t pos = x->list_begin[c]; pos < x->list_begin[c + 1]; ++pos) {
            const size_t slot = static_cast<size_t>(x->tile_begin[c]) * 32 + (pos - x->list_begin[c]);
            uint8_t* row = rows.data() + pos * stride;
            for (size_t q = 0; q < nc; ++q) {
                std::memcpy(row + 8 * q, &cf[q * x->nslots + slot], 4);
                std::memcpy(row + 8 * q + 4, &hh[q * x->nslots + slot], 4);
            }
            uint8_t* cur = row + 8 * nc;
            for (const auto& run : x->runs) {
                if (run.bits == 0) continue;
                const int b = run.bits;
                for (int blk = 0; blk < run.len / 8; ++blk, cur += b) {
                    auto put = [&](int at, int width, uint32_t v) {
                        for (int t = 0; t < width; ++t)
                            if ((v >> t) & 1u) cur[(at + t) >> 3] |= static_cast<uint8_t>(1u << ((at + t) & 7));
                    };
                    const uint16_t* d = dg.data() + pos * pd + run.off + blk * 8;
                    for (int i = 0; i < 7; ++i) put(b * i, b, d[i]);
                    put(b * 7, b - 1, static_cast<uint32_t>(d[7]) >> 1);
                    put(8 * b - 1, 1, br[pos * B + run.off / 8 + blk]);
                }
            }
        }
    std::unique_ptr<std::FILE, int (*)(std::FILE*)> f(std::fopen(path, "wb"), &std::fclose);
    if (!f) fail(E8QC_EIO, std::string("Me8qIndex::Save: cannot write ") + path);
    bool ok = true;
    auto wr = [&](const void* p, size_t bytes) {
        if (bytes && std::fwrite(p, 1, bytes, f.get()) != bytes) ok = false;
    };
    wr("ME8QIDXX", 8);
    const uint64_t hdr[5] = {n, x->dim, pd, nlist, stride};
    wr(hdr, sizeof(hdr));
    wr(&x->avg_bits, 4);
    int32_t flags[4] = {0, x->max_bits, x->drop_energy ? 1 : 0, 0};
    std::memcpy(&flags[3], &x->prune_alpha, 4);
    wr(flags, sizeof(flags));
    const uint64_t nplan = x->plan.size();
    wr(&nplan, 8);
    for (const auto& seg : x->plan) {
        const uint64_t len = seg.first;
        const int32_t bits = seg.second;
        wr(&len, 8);
        wr(&bits, 4);
    }
    wr(x->cen_host.data(), x->cen_host.size() * 4);
    wr(x->ids_compact.data(), n * 4);
    wr(x->list_begin.data(), (nlist + 1) * 8);
    std::vector<uint64_t> byte_begin(nlist + 1);
    for (size_t c = 0; c <= nlist; ++c) byte_begin[c] = x->list_begin[c] * stride;
    wr(byte_begin.data(), byte_begin.size() * 8);
    wr(rows.data(), rows.size());
    wr(&x->rot_seed, 8);
    const uint64_t n_rot = nc;
    wr(&n_rot, 8);
    size_t so = 0;
    for (const auto& run : x->runs) {
        if (run.bits == 0) continue;
        const uint64_t bytes = rotator_signs(static_cast<size_t>(run.len), 0).size();
        if (so + bytes > x->signs_host.size()) fail(E8QC_ESTATE, "rotator signs missing");
        wr(&bytes, 8);
        wr(x->signs_host.data() + so, bytes);
        so += bytes;
    }
    if (!ok) fail(E8QC_EIO, std::string("Me8qIndex::Save: write failed ") + path);
}

uint64_t tune_key(int mode, size_t nq, size_t np) {
    auto lg = [](size_t v) {
        uint64_t l = 0;
        while ((size_t(1) << (l + 1)) <= v) ++l;
        return l;
    };
    return (static_cast<uint64_t>(mode) << 16) | (lg(nq) << 8) | lg(np);
}

// The stored setting of a batch shape (schedule 0 and 6 stages when none) into ws.
void apply_stored(e8qc_me8q* x, Workspace& ws, int mode, size_t nq, size_t np) {
    std::lock_guard<std::mutex> lock(x->tune_mu);
    auto it = x->tuned.find(tune_key(mode, nq, np));
    ws.sched = it == x->tuned.end() ? 0 : it->second.first;
    ws.stages = it == x->tuned.end() ? 6 : it->second.second;
}

void check_mode(int mode) {
    if (mode != E8QC_MODE_BATCHED && mode != E8QC_MODE_PRECISION)
        fail(E8QC_EINVAL, "ME8Q search modes are E8QC_MODE_BATCHED and E8QC_MODE_PRECISION");
}

// The direct search also takes E8QC_MODE_PRUNED (the reference's production
// search; uniform k and nprobe).
void check_search_mode(int mode) {
    if (mode != E8QC_MODE_PRUNED) check_mode(mode);
}

// The pruned search's fast layout, built on first use (synchronises s):
// plane, fits and banks from the code streams (me8q_fast.cu).
void ensure_fast(e8qc_me8q* x, cudaStream_t s) {
    if (x->f_plane.p) return;
    std::vector<Me8qFastRun> fr;
    int blk0 = 0;
    std::vector<float> lev_host;
    for (const auto& r : x->runs) {
        if (r.bits == 0) continue;
        Me8qFastRun f{};
        f.off = r.off;
        f.len = r.len;
        f.bits = r.bits;
        f.word0 = r.word0;
        f.blk0 = blk0;
        blk0 += r.len / 8;
        // ClassModelOf (me8q_codec.cpp:235-262): pbar[c] = mean of the float
        // levels of both branches whose top bit is c, summed in fp64
        const int q = 1 << r.bits, half = q >> 1;
        double sums[2] = {0.0, 0.0};
        for (int c = 0; c < 2; ++c)
            for (int br = 0; br < 2; ++br) {
                const std::vector<double> lv = branch_levels(r.bits, br);
                for (int d = c * half; d < (c + 1) * half; ++d) sums[c] += static_cast<double>(static_cast<float>(lv[d]));
            }
        f.p0 = static_cast<float>(sums[0] / static_cast<double>(2 * half));
        f.p1 = static_cast<float>(sums[1] / static_cast<double>(2 * half));
        fr.push_back(f);
    }
    // level-table offsets as the code streams' chunks hold them
    for (auto& f : fr)
        for (const auto& c : x->chunks)
            if (c.bits == f.bits) {
                f.lev = c.lev;
                break;
            }
    Me8qFast& F = x->fast;
    F = Me8qFast{};
    F.nrun = static_cast<int>(fr.size());
    F.cols = blk0;
    F.colw = (blk0 + 3) / 4;
    if (F.nrun > kFastMaxRuns || F.cols > kFastMaxCols)
        fail(E8QC_EINVAL, "the ME8Q pruned search supports at most 512 coded blocks and 16 coded runs");
    const size_t nr = std::max<size_t>(1, fr.size());
    if (fr.empty()) fr.push_back(Me8qFastRun{});
    x->f_runs.upload(fr.data(), fr.size() * sizeof(Me8qFastRun), s);
    x->f_plane.alloc(std::max<size_t>(1, x->ntiles * static_cast<size_t>(F.colw) * 32 * 4));
    x->f_gain.alloc(nr * std::max<size_t>(1, x->nslots) * 4);
    x->f_vpc.alloc(nr * std::max<size_t>(1, x->nslots) * 4);
    x->f_bank.alloc(std::max<size_t>(1, x->ntiles) * nr * 96);
    x->f_scl.alloc(std::max<size_t>(1, x->ntiles) * nr * 32);
    x->f_rcn2.alloc(std::max<size_t>(1, x->nlist) * nr * 8);
    F.runs = x->f_runs.as<Me8qFastRun>();
    F.plane = x->f_plane.as<uint32_t>();
    F.gain = x->f_gain.as<float>();
    F.vpc = x->f_vpc.as<float>();
    F.bank = x->f_bank.as<uint8_t>();
    F.scl = x->f_scl.as<float>();
    F.rc_n2 = x->f_rcn2.as<double>();
    DevBuf perp;
    perp.alloc(nr * std::max<size_t>(1, x->nslots) * 4);
    fill_view(x);
    launch_me8q_fast_build(x->view, F, x->f_plane.as<uint32_t>(), x->f_gain.as<float>(), x->f_vpc.as<float>(),
                           perp.as<float>(), x->f_bank.as<uint8_t>(), x->f_scl.as<float>(), x->f_rcn2.as<double>(), s);
    E8QC_CUDA(cudaStreamSynchronize(s));
}

// The precision proxy plane, built on first use (synchronises s).
void ensure_proxy(e8qc_me8q* x, cudaStream_t s) {
    if (x->proxy.p) return;
    x->proxy.alloc(proxy_plane_bytes(x->view.base, x->ntiles));
    E8QC_CUDA(cudaMemsetAsync(x->proxy.p, 0, x->proxy.bytes, s));
    x->sigma.alloc(std::max<size_t>(1, x->nslots) * 4);
    fill_view(x);
    launch_me8q_proxy(x->view, static_cast<int>(x->ntiles), static_cast<unsigned char*>(x->proxy.p),
                      x->sigma.as<float>(), s);
    E8QC_CUDA(cudaStreamSynchronize(s));
}

// Proxy rows one query can need: the tiles of its np largest lists.
size_t max_rows(const e8qc_me8q* x, size_t np) {
    return static_cast<size_t>(x->tiles_prefix[std::min(np, x->nlist)]) * 32;
}

// Rotate nq device queries and run the grouped exact scan (batched) or the
// int8 tensor-core candidates + exact rescoring (precision); no host
// synchronisation (k_arr / np_arr may be NULL for uniform k / nprobe).
uint64_t enqueue_search(e8qc_me8q* x, Workspace& ws, int mode, const float* q_dev, size_t nq, const uint32_t* k_arr,
                        const uint32_t* np_arr, size_t k, size_t np, size_t out_stride, uint32_t* ids_d, float* d_d,
                        cudaStream_t s) {
    ws.ensure_queries(nq, x->pd);
    ws.ensure_err();
    launch_me8q_prep(q_dev, x->dim, static_cast<int>(x->dim), static_cast<int>(x->pd), nullptr, nullptr, x->view, 0,
                     nq, ws.rq.as<float>(), nullptr, nullptr, s);
    if (mode == E8QC_MODE_PRUNED) {
        if (!x->f_plane.p) fail(E8QC_ESTATE, "the ME8Q fast layout is not built");
        if (k_arr || np_arr) fail(E8QC_EINVAL, "the ME8Q pruned search takes a uniform k and nprobe");
        const float alpha = x->prune_alpha > 0.0F ? x->prune_alpha : 1.0F;
        const float lambda = ortho_quantile(static_cast<double>(alpha), std::max<size_t>(4 * k, 32));
        if (x->fast.nrun == 0) fail(E8QC_EINVAL, "the ME8Q pruned search needs at least one coded run");
        return 1 + static_cast<uint64_t>(me8q_pruned_search(x->view, x->fast, ws, ws.rq.as<float>(), nq, k, np,
                                                            lambda, out_stride, ids_d, d_d, s));
    }
    if (mode == E8QC_MODE_PRECISION) {
        if (!x->view.base.proxy) fail(E8QC_ESTATE, "the ME8Q proxy plane is not built");
        return 1 + static_cast<uint64_t>(precision_search(x->view.base, ws, ws.rq.as<float>(), nq, k_arr, np_arr, k,
                                                          np, out_stride, ids_d, d_d, max_rows(x, np), s, &x->view));
    }
    return 1 + static_cast<uint64_t>(me8q_grouped_search(x->view, ws, ws.rq.as<float>(), nq, k_arr, np_arr, k, np,
                                                         out_stride, ids_d, d_d, s));
}

class Me8qTarget final : public SearchTarget {
   public:
    explicit Me8qTarget(e8qc_me8q* x) : x_(x) {
        require_built(x, "serve");
        dim = x->dim;
        nlist = x->nlist;
        device = x->device;
    }
    void check_mode(int mode) const override { ::check_mode(mode); }
    void prepare(int mode) override {
        if (mode != E8QC_MODE_PRECISION) return;
        std::lock_guard<std::mutex> lock(x_->mu);
        DeviceGuard g(x_->device);
        ensure_proxy(x_, nullptr);
    }
    size_t bytes(int mode, size_t nq, size_t k_max, size_t np_max) const override {
        const size_t np = std::min(np_max, x_->nlist), nl = x_->nlist, pd = x_->pd;
        const size_t npairs = nq * np;
        const size_t align = mode == E8QC_MODE_PRECISION ? 8 : 1;
        const size_t pslots = npairs + (align - 1) * nl;
        size_t b = nq * (x_->dim * 4 + pd * 4 + k_max * 8 + 8);  // queries, rotated queries, results, k/nprobe
        b += nq * nl * 8 + nq * 4;                                // route keys, norms
        b += npairs * 12 + pslots * 8 + nl * 12;                  // probes, d2, positions; pair rows; counters
        b += (npairs / 64 + nl + 1) * 16 + 32;                    // work items
        if (mode == E8QC_MODE_PRECISION) {
            const size_t rows_q = max_rows(x_, np);
            b += nq * (pd + 12) + nl * 8;            // int8 queries, scales, row bases
            b += precision_row_scratch(nq, rows_q);  // proxy rows of one chunk
            b += ((pslots + 7) / 8 * 8 + 128) * pd;  // gathered int8 query rows
        } else {
            b += npairs * k_max * 8;  // per-pair partial top-k
        }
        return b;
    }
    uint64_t enqueue(Workspace& ws, int mode, const float* q_dev, size_t nq, const uint32_t* k_dev,
                     const uint32_t* np_dev, size_t k_max, size_t np_max, uint32_t* ids_dev, float* d_dev,
                     cudaStream_t s, bool apply_tuned) override {
        const size_t np = std::min(np_max, x_->nlist);
        if (apply_tuned) apply_stored(x_, ws, mode, nq, np);
        return enqueue_search(x_, ws, mode, q_dev, nq, k_dev, np_dev, k_max, np, k_max, ids_dev, d_dev, s);
    }
    // The work-queue order (longest list first / list id order) and, in
    // precision mode, the scan's ring depth (6, 4, 8 stages), timed on nq
    // synthetic rotated queries (mixtures of two lists' rotated centroids).
    void autotune(Workspace& ws, int mode, size_t nq, size_t k, size_t np, cudaStream_t s, int* sched,
                  int* stages) override {
        np = std::min(np, x_->nlist);
        DevBuf rq, ids, d;
        rq.alloc(nq * x_->pd * 4);
        ids.alloc(nq * k * 4);
        d.alloc(nq * k * 4);
        launch_synth_queries(x_->view.base, static_cast<int>(nq), 0x5EEDull, rq.as<float>(), s);
        ws.ensure_err();
        cudaEvent_t e0, e1;
        E8QC_CUDA(cudaEventCreate(&e0));
        E8QC_CUDA(cudaEventCreate(&e1));
        struct Ev {
            cudaEvent_t a, b;
            ~Ev() {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } ev{e0, e1};
        auto run = [&] {
            if (mode == E8QC_MODE_PRECISION)
                precision_search(x_->view.base, ws, rq.as<float>(), nq, nullptr, nullptr, k, np, k,
                                 ids.as<uint32_t>(), d.as<float>(), max_rows(x_, np), s, &x_->view);
            else
                me8q_grouped_search(x_->view, ws, rq.as<float>(), nq, nullptr, nullptr, k, np, k, ids.as<uint32_t>(),
                                    d.as<float>(), s);
        };
        const int stage_opts[3] = {6, 4, 8};
        const int nst = mode == E8QC_MODE_PRECISION ? 3 : 1;
        std::pair<int, int> best{0, 6};
        double best_ms = 1e30;
        for (int sc = 0; sc < 2; ++sc) {
            for (int si = 0; si < nst; ++si) {
                ws.sched = sc;
                ws.stages = stage_opts[si];
                run();  // warm-up: sizes buffers, sets kernel attributes
                E8QC_CUDA(cudaEventRecord(e0, s));
                for (int r = 0; r < 3; ++r) run();
                E8QC_CUDA(cudaEventRecord(e1, s));
                ws.check_error(s);
                float ms = 0.0f;
                E8QC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best_ms) {
                    best_ms = ms;
                    best = {sc, stage_opts[si]};
                }
            }
        }
        ws.sched = best.first;
        ws.stages = best.second;
        {
            std::lock_guard<std::mutex> lock(x_->tune_mu);
            x_->tuned[tune_key(mode, nq, np)] = best;
        }
        *sched = best.first;
        *stages = best.second;
    }
    void stored_tuning(Workspace& ws, int mode, size_t nq, size_t np) override {
        apply_stored(x_, ws, mode, nq, std::min(np, x_->nlist));
    }

   private:
    e8qc_me8q* x_;
};

}  // namespace

namespace e8qc {
std::shared_ptr<SearchTarget> me8q_target(e8qc_me8q* x) { return std::make_shared<Me8qTarget>(x); }
}  // namespace e8qc

extern "C" {

int e8qc_me8q_allocate(const float* var_padded, size_t padded_dim, float avg_bits, int max_bits,
                       double extra_budget_bits, size_t* lens, int* bits, size_t cap, size_t* count) {
    return guarded([&] {
        if (!var_padded || !count) fail(E8QC_EINVAL, "null argument");
        if (padded_dim == 0 || padded_dim % kSegDim != 0) fail(E8QC_EINVAL, "padded_dim must be a multiple of 64");
        if (!(avg_bits > 0.0F)) fail(E8QC_EINVAL, "avg_bits must be positive");
        if (max_bits < 1 || max_bits > kMaxBitsMe8q) fail(E8QC_EINVAL, "max_bits must be in [1, 13]");
        const std::vector<float> var(var_padded, var_padded + padded_dim);
        const Plan plan = allocate(var, padded_dim, avg_bits, max_bits, extra_budget_bits);
        *count = plan.size();
        for (size_t i = 0; i < plan.size() && i < cap; ++i) {
            if (lens) lens[i] = plan[i].first;
            if (bits) bits[i] = plan[i].second;
        }
    });
}

int e8qc_me8q_parse_plan(const char* spec, size_t padded_dim, size_t* lens, int* bits, size_t cap, size_t* count) {
    return guarded([&] {
        if (!spec || !count) fail(E8QC_EINVAL, "null argument");
        const Plan plan = parse_plan(spec, padded_dim);
        *count = plan.size();
        for (size_t i = 0; i < plan.size() && i < cap; ++i) {
            if (lens) lens[i] = plan[i].first;
            if (bits) bits[i] = plan[i].second;
        }
    });
}

int e8qc_me8q_create(int device, size_t dim, float avg_bits, uint64_t seed, e8qc_me8q** out) {
    return guarded([&] {
        if (!out) fail(E8QC_EINVAL, "null output");
        if (dim == 0) fail(E8QC_EINVAL, "dim must be positive");
        if (dim > 16384) fail(E8QC_EINVAL, "dim must be <= 16384");
        if (!(avg_bits > 0.0F)) fail(E8QC_EINVAL, "avg_bits must be positive");
        host_alloc_point();
        int ndev = 0;
        E8QC_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) fail(E8QC_EINVAL, "no such CUDA device");
        auto* x = new e8qc_me8q();
        x->device = device;
        x->dim = dim;
        x->pd = (dim + kSegDim - 1) / kSegDim * kSegDim;
        x->avg_bits = avg_bits;
        x->seed = seed;
        x->ws.device = device;
        *out = x;
    });
}

int e8qc_me8q_destroy(e8qc_me8q* x) {
    return guarded([&] {
        if (!x) return;
        DeviceGuard g(x->device);
        delete x;
    });
}

int e8qc_me8q_build(e8qc_me8q* x, const float* data, size_t n, const float* centroids, size_t nlist,
                    const uint32_t* cluster_ids, const e8qc_me8q_build_opts* opts, void* stream) {
    return guarded([&] {
        if (!x) fail(E8QC_EINVAL, "null index");
        if (!data || !centroids || !cluster_ids || n == 0 || nlist == 0) fail(E8QC_EINVAL, "Me8qIndex::Build: empty input");
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        x->built = false;
        build(x, data, n, centroids, nlist, cluster_ids, opts, static_cast<cudaStream_t>(stream));
    });
}

int e8qc_me8q_load(int device, const char* path, e8qc_me8q** out) {
    return guarded([&] {
        if (!out) fail(E8QC_EINVAL, "null output");
        *out = nullptr;
        if (!path) fail(E8QC_EINVAL, "null path");
        // the dimension comes from the file header (offset 16, after magic and n)
        uint64_t dim = 0;
        {
            std::unique_ptr<std::FILE, int (*)(std::FILE*)> f(std::fopen(path, "rb"), &std::fclose);
            if (!f) fail(E8QC_EIO, std::string("Me8qIndex::Load: cannot read ") + path);
            unsigned char head[24];
            if (std::fread(head, 1, 24, f.get()) != 24) fail(E8QC_EIO, "Me8qIndex::Load: short read (header)");
            if (std::memcmp(head, "ME8QIDXX", 8) != 0) fail(E8QC_EIO, std::string("Me8qIndex::Load: bad magic ") + path);
            std::memcpy(&dim, head + 16, 8);
        }
        if (dim == 0 || dim > 16384) fail(E8QC_EIO, "Me8qIndex::Load: corrupt header");
        e8qc_me8q* x = nullptr;
        const int rc = e8qc_me8q_create(device, static_cast<size_t>(dim), 4.0f, 0, &x);
        if (rc != E8QC_OK) fail(rc, std::string(e8qc_last_error()));
        std::unique_ptr<e8qc_me8q, int (*)(e8qc_me8q*)> hold(x, &e8qc_me8q_destroy);
        {
            std::lock_guard<std::mutex> lock(x->mu);
            DeviceGuard g(x->device);
            load_me8q_file(x, path, nullptr);
        }
        *out = hold.release();
    });
}

int e8qc_me8q_save(e8qc_me8q* x, const char* path) {
    return guarded([&] {
        require_built(x, "save");
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        save_me8q_file(x, path, nullptr);
    });
}

int e8qc_me8q_search(e8qc_me8q* x, const float* queries, size_t nq, size_t k, size_t nprobe, uint32_t* out_ids,
                     float* out_dists, e8qc_stats* stats, void* stream) {
    return e8qc_me8q_search_mode(x, queries, nq, k, nprobe, E8QC_MODE_BATCHED, out_ids, out_dists, stats, stream);
}

int e8qc_me8q_search_mode(e8qc_me8q* x, const float* queries, size_t nq, size_t k, size_t nprobe, int mode,
                          uint32_t* out_ids, float* out_dists, e8qc_stats* stats, void* stream) {
    return guarded([&] {
        require_built(x, "search");
        check_search_mode(mode);
        if (k == 0) fail(E8QC_EINVAL, "k must be positive");
        if (k > static_cast<size_t>(kMaxK)) fail(E8QC_EINVAL, "k must be <= 128");
        if (nprobe == 0) fail(E8QC_EINVAL, "nprobe must be positive");
        if (nq == 0) return;
        if (!queries || !out_ids) fail(E8QC_EINVAL, "null buffer");
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t np = std::min(nprobe, x->nlist);
        Workspace& ws = x->ws;
        const float* qd = queries;
        if (!is_device_ptr(queries)) {
            ws.stage_q.ensure(nq * x->dim * 4);
            E8QC_CUDA(cudaMemcpyAsync(ws.stage_q.p, queries, nq * x->dim * 4, cudaMemcpyHostToDevice, s));
            qd = ws.stage_q.as<float>();
        }
        const bool ids_dev = is_device_ptr(out_ids), d_dev = out_dists && is_device_ptr(out_dists);
        uint32_t* ids_d = out_ids;
        float* d_d = out_dists;
        if (!ids_dev) {
            ws.stage_ids.ensure(nq * k * 4);
            ids_d = ws.stage_ids.as<uint32_t>();
        }
        if (!d_dev) {
            ws.stage_d.ensure(nq * k * 4);
            d_d = ws.stage_d.as<float>();
        }
        if (mode == E8QC_MODE_PRECISION) ensure_proxy(x, s);
        if (mode == E8QC_MODE_PRUNED) ensure_fast(x, s);
        apply_stored(x, ws, mode, nq, np);
        const uint64_t launches = enqueue_search(x, ws, mode, qd, nq, nullptr, nullptr, k, np, k, ids_d, d_d, s);
        if (!ids_dev) E8QC_CUDA(cudaMemcpyAsync(out_ids, ids_d, nq * k * 4, cudaMemcpyDeviceToHost, s));
        if (out_dists && !d_dev) E8QC_CUDA(cudaMemcpyAsync(out_dists, d_d, nq * k * 4, cudaMemcpyDeviceToHost, s));
        ws.check_error(s);
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            uint64_t cntv[2] = {0, 0};
            if (mode == E8QC_MODE_PRUNED) {
                E8QC_CUDA(cudaMemcpyAsync(cntv, ws.f_counts.p, 16, cudaMemcpyDeviceToHost, s));
            } else {
                E8QC_CUDA(cudaMemcpyAsync(cntv, ws.b_nitems.as<uint32_t>() + 2, 16, cudaMemcpyDeviceToHost, s));
                cntv[1] = cntv[0];
            }
            E8QC_CUDA(cudaStreamSynchronize(s));
            stats->candidates = cntv[0];
            stats->survivors = cntv[1];
            stats->launches = launches;
        }
    });
}

int e8qc_me8q_search_ragged(e8qc_me8q* x, const float* queries, size_t nq, const uint32_t* k, const uint32_t* nprobe,
                            size_t k_max, int mode, uint32_t* out_ids, float* out_dists, void* stream) {
    return guarded([&] {
        require_built(x, "search");
        check_mode(mode);
        if (nq == 0) return;
        if (!queries || !k || !nprobe || !out_ids) fail(E8QC_EINVAL, "null buffer");
        if (k_max == 0 || k_max > static_cast<size_t>(kMaxK)) fail(E8QC_EINVAL, "k_max must be in [1, 128]");
        if (is_device_ptr(k) || is_device_ptr(nprobe)) fail(E8QC_EINVAL, "k and nprobe must be host arrays");
        size_t np_max = 1;
        std::vector<uint32_t> kk(nq), nn(nq);
        for (size_t i = 0; i < nq; ++i) {
            if (k[i] == 0 || k[i] > k_max) fail(E8QC_EINVAL, "k must be in [1, k_max]");
            if (nprobe[i] == 0) fail(E8QC_EINVAL, "nprobe must be positive");
            kk[i] = k[i];
            nn[i] = static_cast<uint32_t>(std::min<size_t>(nprobe[i], x->nlist));
            np_max = std::max<size_t>(np_max, nn[i]);
        }
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        Workspace& ws = x->ws;
        const float* qd = queries;
        if (!is_device_ptr(queries)) {
            ws.stage_q.ensure(nq * x->dim * 4);
            E8QC_CUDA(cudaMemcpyAsync(ws.stage_q.p, queries, nq * x->dim * 4, cudaMemcpyHostToDevice, s));
            qd = ws.stage_q.as<float>();
        }
        ws.stage_k.ensure(nq * 4);
        ws.stage_np.ensure(nq * 4);
        E8QC_CUDA(cudaMemcpyAsync(ws.stage_k.p, kk.data(), nq * 4, cudaMemcpyHostToDevice, s));
        E8QC_CUDA(cudaMemcpyAsync(ws.stage_np.p, nn.data(), nq * 4, cudaMemcpyHostToDevice, s));
        const bool ids_dev = is_device_ptr(out_ids), d_dev = out_dists && is_device_ptr(out_dists);
        uint32_t* ids_d = out_ids;
        float* d_d = out_dists;
        if (!ids_dev) {
            ws.stage_ids.ensure(nq * k_max * 4);
            ids_d = ws.stage_ids.as<uint32_t>();
        }
        if (!d_dev) {
            ws.stage_d.ensure(nq * k_max * 4);
            d_d = ws.stage_d.as<float>();
        }
        if (mode == E8QC_MODE_PRECISION) ensure_proxy(x, s);
        apply_stored(x, ws, mode, nq, np_max);
        enqueue_search(x, ws, mode, qd, nq, ws.stage_k.as<uint32_t>(), ws.stage_np.as<uint32_t>(), k_max, np_max, k_max,
                       ids_d, d_d, s);
        if (!ids_dev) E8QC_CUDA(cudaMemcpyAsync(out_ids, ids_d, nq * k_max * 4, cudaMemcpyDeviceToHost, s));
        if (out_dists && !d_dev)
            E8QC_CUDA(cudaMemcpyAsync(out_dists, d_d, nq * k_max * 4, cudaMemcpyDeviceToHost, s));
        ws.check_error(s);
    });
}

int e8qc_me8q_estimate(e8qc_me8q* x, const float* query, uint32_t id, float* out) {
    return guarded([&] {
        require_built(x, "estimate");
        if (!query || !out) fail(E8QC_EINVAL, "null buffer");
        std::lock_guard<std::mutex> lock(x->mu);
        if (x->inv_pos.size() != x->n) {
            x->inv_pos.assign(x->n, 0xFFFFFFFFu);
            for (size_t i = 0; i < x->n; ++i) x->inv_pos[x->ids_compact[i]] = static_cast<uint32_t>(i);
        }
        if (id >= x->n || x->inv_pos[id] == 0xFFFFFFFFu) fail(E8QC_ERANGE, "Me8qIndex::Estimate: unknown id");
        const uint64_t pos = x->inv_pos[id];
        const size_t c = static_cast<size_t>(
            std::upper_bound(x->list_begin.begin() + 1, x->list_begin.end(), pos) - x->list_begin.begin() - 1);
        const uint32_t slot = x->tile_begin[c] * 32 + static_cast<uint32_t>(pos - x->list_begin[c]);
        DeviceGuard g(x->device);
        cudaStream_t s = nullptr;
        std::vector<float> qpad(x->pd, 0.0f);
        if (is_device_ptr(query)) E8QC_CUDA(cudaMemcpy(qpad.data(), query, x->dim * 4, cudaMemcpyDeviceToHost));
        else std::memcpy(qpad.data(), query, x->dim * 4);
        DevBuf qp, rq, o;
        qp.upload(qpad.data(), x->pd * 4, s);
        rq.alloc(x->pd * 4);
        o.alloc(4);
        launch_me8q_prep(qp.as<float>(), x->pd, static_cast<int>(x->pd), static_cast<int>(x->pd), nullptr, nullptr, x->view,
                         0, 1, rq.as<float>(), nullptr, nullptr, s);
        launch_me8q_estimate(x->view, rq.as<float>(), qp.as<float>(), x->cen_pad.as<float>(), static_cast<uint32_t>(c), slot,
                             o.as<float>(), s);
        E8QC_CUDA(cudaMemcpy(out, o.p, 4, cudaMemcpyDeviceToHost));
    });
}

int e8qc_me8q_info(const e8qc_me8q* x, e8qc_me8q_meta* out) {
    return guarded([&] {
        if (!x || !out) fail(E8QC_EINVAL, "null argument");
        e8qc_me8q_meta in{};
        in.n = x->n;
        in.dim = x->dim;
        in.padded_dim = x->pd;
        in.nlist = x->nlist;
        in.nruns = x->plan.size();
        in.ncoded = static_cast<size_t>(x->ncoded);
        in.route_dim = static_cast<size_t>(x->route_dim);
        in.bytes_per_vector = x->bytes_per_vector;
        in.bits_per_dim = x->dim ? 8.0 * static_cast<double>(x->bytes_per_vector) / static_cast<double>(x->dim) : 0.0;
        in.memory_bytes = x->memory_bytes();
        in.avg_bits = x->avg_bits;
        in.is_built = x->built ? 1 : 0;
        *out = in;
    });
}

int e8qc_me8q_plan(const e8qc_me8q* x, size_t* lens, int* bits, size_t cap, size_t* count) {
    return guarded([&] {
        if (!x || !count) fail(E8QC_EINVAL, "null argument");
        *count = x->plan.size();
        for (size_t i = 0; i < x->plan.size() && i < cap; ++i) {
            if (lens) lens[i] = x->plan[i].first;
            if (bits) bits[i] = x->plan[i].second;
        }
    });
}

int e8qc_me8q_get_ids(const e8qc_me8q* x, uint32_t* out) {
    return guarded([&] {
        require_built(x, "get_ids");
        if (!out) fail(E8QC_EINVAL, "null buffer");
        std::memcpy(out, x->ids_compact.data(), x->n * 4);
    });
}

int e8qc_me8q_export_codes(e8qc_me8q* x, uint16_t* digits, uint8_t* branch, float* coef, float* h2) {
    return guarded([&] {
        require_built(x, "export_codes");
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = nullptr;
        const size_t n = x->n, pd = x->pd;
        if (digits || branch) {
            DevBuf dd, bb;
            dd.alloc(n * pd * 2);
            bb.alloc(n * (pd / 8));
            launch_me8q_decode(x->view, static_cast<int>(x->ntiles), x->list_of_tile_d.as<uint32_t>(),
                               x->list_begin_d.as<uint64_t>(), static_cast<int>(pd), dd.as<uint16_t>(), bb.as<uint8_t>(), s);
            if (digits) E8QC_CUDA(cudaMemcpy(digits, dd.p, n * pd * 2, cudaMemcpyDeviceToHost));
            if (branch) E8QC_CUDA(cudaMemcpy(branch, bb.p, n * (pd / 8), cudaMemcpyDeviceToHost));
        }
        if (coef || h2) {
            const size_t nc = static_cast<size_t>(x->ncoded);
            std::vector<float> cf(nc * x->nslots), hh(nc * x->nslots);
            if (nc) {
                E8QC_CUDA(cudaMemcpy(cf.data(), x->coef.p, cf.size() * 4, cudaMemcpyDeviceToHost));
                E8QC_CUDA(cudaMemcpy(hh.data(), x->h2.p, hh.size() * 4, cudaMemcpyDeviceToHost));
            }
            for (size_t c = 0; c < x->nlist; ++c)
                for (uint64_t p = x->list_begin[c]; p < x->list_begin[c + 1]; ++p) {
                    const size_t slot = static_cast<size_t>(x->tile_begin[c]) * 32 + (p - x->list_begin[c]);
                    for (size_t q = 0; q < nc; ++q) {
                        if (coef) coef[p * nc + q] = cf[q * x->nslots + slot];
                        if (h2) h2[p * nc + q] = hh[q * x->nslots + slot];
                    }
                }
        }
    });
}

}  // extern "C"
