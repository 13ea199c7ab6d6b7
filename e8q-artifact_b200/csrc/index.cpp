// C ABI of libe8qcuda.so (include/e8qc.h): the E8Q index object, its device
// memory, the build orchestration and the search/estimate entry points.
//
// Mirrors the reference's E8qIndex (include/e8qlib/index/e8q.hpp:121-187,
// python_bindings/e8q_bindings.cpp) with the data held in HBM and every
// per-vector step run by the kernels in search_kernels.cu / build_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <atomic>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "e8qc.h"
#include "internal.h"
#include "scan_plain.h"
#include "io_e8ax.h"
#include "precision.h"
#include "pruned.h"
#include "serve_target.h"
#include "workspace.h"

namespace e8qc {

namespace {
thread_local std::string g_last_error;
}

void fail(int code, const std::string& msg) { throw Error{code, msg}; }

namespace {
std::atomic<int> g_fail_host_allocs{0};  // injected host-allocation failures left
}  // namespace

void host_alloc_point() {
    for (int left = g_fail_host_allocs.load(); left > 0;)
        if (g_fail_host_allocs.compare_exchange_weak(left, left - 1)) throw std::bad_alloc();
}

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? E8QC_ENOMEM : E8QC_ECUDA;
        fail(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void set_last_error(const std::string& s) { g_last_error = s; }
const char* last_error() { return g_last_error.c_str(); }

bool is_device_ptr(const void* p) {
    if (p == nullptr) return false;
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device memory of `device` itself (or managed memory, reachable from every
// device): a buffer on another GPU would be dereferenced through a peer
// mapping that may not exist.
bool is_device_ptr_on(const void* p, int device) {
    if (p == nullptr) return false;
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

std::vector<uint8_t> rotator_signs(size_t dim, uint64_t seed) {
    // FhtKac4Rotator(dim, seed) (src/utils/rotator.cpp:13-28): one byte per
    // draw of mt19937_64; a uniform [0, 255] draw from a full 64-bit engine
    // is its top byte (multiply-shift reduction, no rejection for 256).
    const size_t pd = (dim + 63) / 64 * 64;
    std::vector<uint8_t> s(4 * pd / 8);
    std::mt19937_64 gen(seed);
    for (auto& b : s) b = static_cast<uint8_t>(gen() >> 56);
    return s;
}

// Grouped-mode searches of host-resident queries from this many queries whose
// shape repeats the previous call's replay a captured graph of that shape.
constexpr size_t kGraphMinQueries = 1024;

// Input staging: device pointers pass through, host data is copied to a
// temporary device buffer on the call's stream.
template <class T>
const T* stage_in(const T* p, size_t count, DevBuf& tmp, cudaStream_t s) {
    if (count == 0 || is_device_ptr(p)) return p;
    tmp.ensure(count * sizeof(T));
    E8QC_CUDA(cudaMemcpyAsync(tmp.p, p, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return static_cast<const T*>(tmp.p);
}

}  // namespace e8qc

using namespace e8qc;

struct e8qc_index {
    int device = 0;
    size_t dim = 0, pd = 0;
    int bits = 0;
    uint64_t seed = 0;
    bool built = false;
    bool disable_prune = false;
    float prune_alpha = 1.0f;
    size_t n = 0, nlist = 0, ntiles = 0;
    int nch = 0, B = 0;
    std::mutex mu;

    std::vector<uint64_t> list_begin;  // nlist+1 compact offsets
    std::vector<uint32_t> tile_begin;  // nlist+1
    std::vector<uint32_t> ids_compact; // n
    std::vector<uint32_t> inv_pos;     // global id -> compact position (lazy)
    std::vector<uint32_t> sorted_tiles_prefix;  // prefix of list tile counts, largest first

    DevBuf signs, mean_rot, cen, cn2, tile_begin_d, list_len_d, codes, g1, h3, ids, tab,
        list_of_tile, list_begin_d, list_order;
    DevBuf ortho;   // built indexes: per slot the scan-bank inputs (base, weight, perp), for saving
    std::vector<uint8_t> banks;  // loaded indexes: the file's 128-byte scan-bank headers, for saving
    DevBuf rowa;     // pruned mode: the coarse plane (rowA bytes per vector), built on its first search
    DevBuf banks_d;  // pruned mode: the 128-byte scan-bank header of every tile
    DevBuf proxy;   // int8 proxy plane of the precision mode, built on its first search
    DevBuf vcodes;  // the codes slot-major, for the precision mode's rescoring (built with the plane)
    // autotuned (schedule, stages) per (mode, log2 batch size, log2 nprobe)
    std::mutex tune_mu;
    std::map<uint64_t, std::pair<int, int>> tuned;
    DevIndex view{};
    Workspace ws;
    bool profiling = false;
    e8qc_profile prof{};
    // fault injection (e8qc_e8q_debug_inject_wait_timeout): plain searches
    // left whose scan waits on a barrier nothing completes, and the bound
    std::atomic<int> inject_waits{0};
    std::atomic<uint32_t> inject_wait_ms{0};

    size_t memory_bytes() const {
        return signs.bytes + mean_rot.bytes + cen.bytes + cn2.bytes + tile_begin_d.bytes +
               list_len_d.bytes + codes.bytes + g1.bytes + h3.bytes + ids.bytes + tab.bytes +
               list_of_tile.bytes + list_begin_d.bytes + list_order.bytes + proxy.bytes + vcodes.bytes +
               ortho.bytes + banks.size() + rowa.bytes + banks_d.bytes;
    }
    // A captured graph of the last repeated batch shape of the grouped modes
    // (search calls from kGraphMinQueries queries whose mode, size, k and
    // nprobe equal the previous call's): later calls of that shape replay it.
    // Declared last, so it is released before the buffers it points into.
    struct GraphKey {
        int mode = -1;
        size_t nq = 0, k = 0, np = 0;
        bool operator==(const GraphKey& o) const { return mode == o.mode && nq == o.nq && k == o.k && np == o.np; }
    };
    std::mutex gmu;
    GraphKey glast, gkey;
    std::shared_ptr<e8qc_plan> gplan;
};

namespace {

// The precision mode's device planes (int8 proxies, slot-major codes), built
// on first use; returns the kernels launched.
int ensure_precision_planes(e8qc_index* x, cudaStream_t s) {
    if (x->view.proxy != nullptr) return 0;
    int launches = 0;
    x->vcodes.alloc(vcodes_bytes(x->view, x->ntiles));
    launches += launch_vcodes(x->view, static_cast<int>(x->ntiles), x->vcodes.as<uint4>(), s);
    x->proxy.alloc(proxy_plane_bytes(x->view, x->ntiles));
    launches += launch_build_proxy(x->view, static_cast<int>(x->ntiles), x->proxy.as<uint4>(), s);
    x->view.vcodes = x->vcodes.as<uint4>();
    x->view.proxy = x->proxy.as<uint4>();
    x->view.proxy_scale = precision_proxy_step(x->view.bits, x->view.pd);
    return launches;
}

}  // namespace

namespace {

struct DeviceGuard {
    int prev = 0;
    explicit DeviceGuard(int d) {
        E8QC_CUDA(cudaGetDevice(&prev));
        if (prev != d) E8QC_CUDA(cudaSetDevice(d));
    }
    ~DeviceGuard() { cudaSetDevice(prev); }
};

template <class F>
int guarded(F&& f) {
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

void require_built(const e8qc_index* x, const char* what) {
    if (x == nullptr) fail(E8QC_EINVAL, "null index");
    if (!x->built) fail(E8QC_ESTATE, std::string("E8qIndex must be built or loaded before ") + what);
}

// Upper bound of the tiles any nprobe lists can hold (sum of the largest).
size_t max_tiles_for(const e8qc_index* x, size_t nprobe) {
    const size_t p = std::min(nprobe, x->nlist);
    return x->sorted_tiles_prefix[p];
}

void plain_search(e8qc_index* x, const float* rq_all, size_t nq, size_t k, size_t nprobe,
                  uint32_t* ids_d, float* d_d, e8qc_stats* st, cudaStream_t s) {
    Workspace& ws = x->ws;
    ws.ensure_route(x->nlist);
    // grid: one CTA per SM (the kernel fills an SM's registers and shared
    // memory) but one, fewer when the largest possible probe set has fewer
    // tiles than that. The scan starts while the routing kernel's last CTA
    // still selects the probes; that CTA's SM is the one left out, so no scan
    // CTA waits for it.
    const size_t max_tiles = max_tiles_for(x, nprobe);
    int sms = 148;
    E8QC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device));
    int grid = static_cast<int>(std::min<size_t>(max_tiles, static_cast<size_t>(std::max(1, sms - 1))));
    grid = std::max(grid, 1);
    const ScanGeo geo =
        plain_scan_geo(x->view, (max_tiles + static_cast<size_t>(grid) - 1) / static_cast<size_t>(grid));
    ws.ensure_scan(static_cast<size_t>(grid));
    RouteWork rw{ws.keys.as<uint64_t>(), ws.probes.as<uint32_t>(), ws.probe_d2.as<float>(),
                 ws.tile_off.as<uint32_t>(), ws.route_counter.as<uint32_t>(),
                 ws.total_tiles.as<uint32_t>(), ws.probe_info.as<uint2>()};
    ScanWork sw{ws.part_d.as<float>(), ws.part_id.as<uint32_t>(), ws.scan_counter.as<uint32_t>(),
                ws.err.as<uint32_t>(), grid};

    uint64_t launches = 0;
    cudaEvent_t er = nullptr, e0 = nullptr, e1 = nullptr;
    std::vector<uint32_t> probes;
    if (x->profiling) {
        E8QC_CUDA(cudaEventCreate(&er));
        E8QC_CUDA(cudaEventCreate(&e0));
        E8QC_CUDA(cudaEventCreate(&e1));
        probes.resize(nprobe);
    }
    for (size_t i = 0; i < nq; ++i) {
        const float* rq = rq_all + i * x->pd;
        if (x->profiling) E8QC_CUDA(cudaEventRecord(er, s));
        launches += launch_route_one(x->view, rq, static_cast<int>(nprobe), rw, s);
        if (x->profiling) E8QC_CUDA(cudaEventRecord(e0, s));
        sw.stuck_ms = 0;
        for (int left = x->inject_waits.load(); left > 0;)
            if (x->inject_waits.compare_exchange_weak(left, left - 1)) {
                sw.stuck_ms = x->inject_wait_ms.load();
                break;
            }
        launches += launch_scan_plain(x->view, rq, rw, static_cast<int>(nprobe), static_cast<int>(k), sw,
                                      geo, ids_d + i * k, d_d + i * k, s);
        if (x->profiling) {
            E8QC_CUDA(cudaEventRecord(e1, s));
            E8QC_CUDA(cudaMemcpyAsync(probes.data(), rw.probes, nprobe * 4, cudaMemcpyDeviceToHost, s));
            E8QC_CUDA(cudaStreamSynchronize(s));
            float ms = 0.0f, rms = 0.0f;
            E8QC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            E8QC_CUDA(cudaEventElapsedTime(&rms, er, e0));
            x->prof.prep_ms += rms;  // the routing launch of this query
            uint64_t cand = 0;
            for (uint32_t c : probes) cand += x->list_begin[c + 1] - x->list_begin[c];
            x->prof.scan_launches += 1;
            x->prof.scan_ms += ms;
            x->prof.candidates += cand;
            x->prof.algo_bytes += cand * (static_cast<uint64_t>(x->bits) * x->pd / 8 + 8);
            x->prof.item_bytes += cand * (static_cast<uint64_t>(x->bits) * x->pd / 8 + 8);
            x->prof.list_vectors += cand;
            x->prof.list_once += cand;
            x->prof.queries += 1;
        }
    }
    if (er) cudaEventDestroy(er);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) st->launches += launches;
}

void scan_class_means(int bits, double w_cls[2]);

// The pruned mode's device planes: the coarse plane (derived from the codes)
// and the scan-bank headers of every tile -- a loaded index's headers as its
// file holds them, a built index's quantised from its bank inputs (the
// reference's WriteOrthoBanks, which its saved files carry). Built on first
// use; returns the kernels launched.
int ensure_pruned_planes(e8qc_index* x, cudaStream_t s) {
    if (x->rowa.p != nullptr) return 0;
    int launches = 0;
    if (!x->banks.empty()) {
        // a loaded file's headers, as read
        if (x->banks.size() != x->ntiles * 128) fail(E8QC_ESTATE, "scan-bank headers do not match the tiles");
        x->banks_d.upload(x->banks.data(), x->banks.size(), s);
    } else if (x->ortho.bytes != 0) {
        // a build's per-slot bank inputs, quantised on the device
        x->banks_d.alloc(std::max<size_t>(1, x->ntiles * 128));
        launches += launch_ortho_banks(x->ortho.as<float>(), x->ids.as<uint32_t>(), static_cast<int>(x->ntiles),
                                       x->banks_d.as<uint8_t>(), s);
    } else {
        fail(E8QC_ESTATE, "index holds no scan banks for the pruned search");
    }
    DevBuf rowa;
    rowa.alloc(x->ntiles * static_cast<size_t>(rowa_chunks(x->B)) * 32 * 16);
    launches += launch_build_rowa(x->view, static_cast<int>(x->ntiles), rowa.as<uint4>(), s);
    E8QC_CUDA(cudaStreamSynchronize(s));
    std::swap(x->rowa.p, rowa.p);
    std::swap(x->rowa.bytes, rowa.bytes);
    return launches;
}

// The reference's production search for a batch: the batched route, then
// per-query u8 LUTs and one warp per query replaying the reference's scan
// with its running heap (pruned.cu, launch_pruned_batch).
void pruned_search(e8qc_index* x, const float* rq_all, size_t nq, size_t k, size_t nprobe, uint32_t* ids_d,
                   float* d_d, e8qc_stats* st, cudaStream_t s) {
    Workspace& ws = x->ws;
    uint64_t launches = static_cast<uint64_t>(ensure_pruned_planes(x, s));
    // route + per-query probes (the batched route; its pair grouping is unused)
    launches += static_cast<uint64_t>(batched_prepare(x->view, ws, rq_all, nq, nullptr, nprobe, 1, 64, 1, s));
    ws.ensure_pruned(nq);
    ws.f_lut.ensure(nq * static_cast<size_t>(x->B) * 32);
    ws.f_qrun.ensure(nq * 16);
    double w_cls[2];
    scan_class_means(x->bits, w_cls);
    PrunedWork pw{};
    pw.stats = ws.pr_stats.as<unsigned long long>();
    pw.thr = ws.pr_thr.as<float>();
    pw.err = ws.err.as<uint32_t>();
    pw.banks = x->banks_d.as<uint8_t>();
    pw.rowa = x->rowa.as<uint4>();
    pw.nrc = rowa_chunks(x->B);
    pw.z = ortho_quantile(static_cast<double>(x->prune_alpha), std::max<size_t>(4 * k, 32));
    pw.w_cls0 = w_cls[0];
    pw.w_cls1 = w_cls[1];
    pw.disable_prune = x->disable_prune ? 1 : 0;
    E8QC_CUDA(cudaMemsetAsync(ws.pr_stats.p, 0, 16, s));
    // the probed rows' coarse values are kept per group of queries, within
    // min(8 GB, a quarter of the free device memory)
    PrunedScratch sc{};
    sc.max_tiles = std::max<size_t>(1, max_tiles_for(x, nprobe));
    const size_t per_q = sc.max_tiles * 32 * 12;
    size_t free_b = 0, total_b = 0;
    E8QC_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = std::min<size_t>(size_t{8} << 30, free_b / 4);
    sc.group = static_cast<int>(std::max<size_t>(1, std::min<size_t>(nq, budget / per_q)));
    ws.p2_toff.ensure(static_cast<size_t>(sc.group) * (nprobe + 1) * 4);
    ws.p2_acc.ensure(static_cast<size_t>(sc.group) * sc.max_tiles * 32 * 4);
    ws.p2_P.ensure(static_cast<size_t>(sc.group) * sc.max_tiles * 32 * 4);
    ws.p2_perp.ensure(static_cast<size_t>(sc.group) * sc.max_tiles * 32 * 4);
    sc.lut8 = ws.f_lut.as<uint8_t>();
    sc.scal = ws.f_qrun.as<float>();
    sc.toff = ws.p2_toff.as<uint32_t>();
    sc.c_acc = ws.p2_acc.as<int>();
    sc.c_P = ws.p2_P.as<float>();
    sc.c_perp = ws.p2_perp.as<float>();
    sc.out_ids = ids_d;
    sc.out_d = d_d;
    launches += static_cast<uint64_t>(launch_pruned_batch(x->view, rq_all, ws.b_probes.as<uint32_t>(),
                                                          ws.b_pd2.as<float>(), static_cast<int>(nq),
                                                          static_cast<int>(nprobe), static_cast<int>(k), pw, sc, s));
    ws.pr_last_nq = nq;
    if (st) {
        unsigned long long cs[2] = {0, 0};
        E8QC_CUDA(cudaMemcpyAsync(cs, ws.pr_stats.p, 16, cudaMemcpyDeviceToHost, s));
        E8QC_CUDA(cudaStreamSynchronize(s));
        st->candidates += cs[0];
        st->survivors += cs[1];
        st->launches += launches;
    }
}

// ---- autotuning of the grouped paths ----
int log2_ceil(size_t v) {
    int b = 0;
    while ((size_t(1) << b) < v) ++b;
    return b;
}
uint64_t tune_key(int mode, size_t nq, size_t np) {
    return (static_cast<uint64_t>(mode) << 32) | (static_cast<uint64_t>(log2_ceil(nq)) << 16) |
           static_cast<uint64_t>(log2_ceil(np));
}
// The tuned (schedule, stages) of this batch shape, or the defaults (0, 6).
void apply_tuning(e8qc_index* x, Workspace& ws, int mode, size_t nq, size_t np) {
    std::lock_guard<std::mutex> lock(x->tune_mu);
    auto it = x->tuned.find(tune_key(mode, nq, np));
    ws.sched = it == x->tuned.end() ? 0 : it->second.first;
    ws.stages = it == x->tuned.end() ? 6 : it->second.second;
}

struct TuneResult {
    int sched, stages;
    double best_ms, default_ms;
};

// Time every (schedule, stages) setting on nq synthetic queries with uniform
// k / nprobe and keep the fastest for this batch shape. Candidate settings
// change only the work order and the scan's ring depth, never the results.
TuneResult autotune_run(e8qc_index* x, Workspace& ws, int mode, size_t nq, size_t k, size_t np, cudaStream_t s) {
    np = std::min(np, x->nlist);
    DevBuf rq, ids, d;
    rq.alloc(nq * x->pd * 4);
    ids.alloc(nq * k * 4);
    d.alloc(nq * k * 4);
    launch_synth_queries(x->view, static_cast<int>(nq), 0x5EEDull, rq.as<float>(), s);
    ws.ensure_err();
    auto run = [&] {
        if (mode == E8QC_MODE_PRECISION)
            precision_search(x->view, ws, rq.as<float>(), nq, nullptr, nullptr, k, np, k, ids.as<uint32_t>(),
                             d.as<float>(), max_tiles_for(x, np) * 32, s);
        else
            batched_search(x->view, ws, rq.as<float>(), nq, nullptr, nullptr, k, np, k, ids.as<uint32_t>(),
                           d.as<float>(), max_tiles_for(x, np), s);
    };
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
    TuneResult best{0, 6, 1e30, 0.0};
    const int nst = mode == E8QC_MODE_PRECISION ? 3 : 1;
    const int stage_opts[3] = {6, 4, 8};
    for (int sched = 0; sched < 2; ++sched) {
        for (int si = 0; si < nst; ++si) {
            ws.sched = sched;
            ws.stages = stage_opts[si];
            run();  // warm-up (sizes buffers, sets kernel attributes)
            E8QC_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < 3; ++r) run();
            E8QC_CUDA(cudaEventRecord(e1, s));
            ws.check_error(s);
            float ms = 0.0f;
            E8QC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            const double t = ms / 3.0;
            if (sched == 0 && si == 0) best.default_ms = t;
            if (t < best.best_ms) best = TuneResult{sched, stage_opts[si], t, best.default_ms};
        }
    }
    ws.sched = best.sched;
    ws.stages = best.stages;
    std::lock_guard<std::mutex> lock(x->tune_mu);
    x->tuned[tune_key(mode, nq, np)] = {best.sched, best.stages};
    return best;
}

// Batched or precision search of nq rotated queries; while profiling, times
// the scan kernel with CUDA events and reads back its pair / vector counters.
uint64_t grouped_search(e8qc_index* x, int mode, const float* rq, size_t nq, const uint32_t* k_arr,
                        const uint32_t* np_arr, size_t k, size_t np, uint32_t* ids_d, float* d_d, cudaStream_t s) {
    Workspace& ws = x->ws;
    if (x->profiling) {
        E8QC_CUDA(cudaEventCreate(&ws.scan_ev0));
        E8QC_CUDA(cudaEventCreate(&ws.scan_ev1));
        if (mode == E8QC_MODE_PRECISION) {
            E8QC_CUDA(cudaEventCreate(&ws.final_ev0));
            E8QC_CUDA(cudaEventCreate(&ws.final_ev1));
            E8QC_CUDA(cudaEventCreate(&ws.prep_ev0));
            E8QC_CUDA(cudaEventCreate(&ws.prep_ev1));
        }
    }
    struct Drop {
        Workspace& w;
        ~Drop() {
            for (cudaEvent_t* e : {&w.scan_ev0, &w.scan_ev1, &w.final_ev0, &w.final_ev1, &w.prep_ev0, &w.prep_ev1}) {
                if (*e) cudaEventDestroy(*e);
                *e = nullptr;
            }
        }
    } drop{ws};
    int launches = 0;
    apply_tuning(x, ws, mode, nq, np);
    if (mode == E8QC_MODE_PRECISION) launches += ensure_precision_planes(x, s);
    if (mode == E8QC_MODE_PRECISION)
        launches += precision_search(x->view, ws, rq, nq, k_arr, np_arr, k, np, k, ids_d, d_d,
                                     max_tiles_for(x, np) * 32, s);
    else
        launches += batched_search(x->view, ws, rq, nq, k_arr, np_arr, k, np, k, ids_d, d_d, max_tiles_for(x, np), s);
    if (x->profiling) {
        uint64_t cnt[3] = {0, 0, 0};
        E8QC_CUDA(cudaMemcpyAsync(cnt, ws.b_nitems.as<uint32_t>() + 2, 24, cudaMemcpyDeviceToHost, s));
        E8QC_CUDA(cudaStreamSynchronize(s));
        float ms = 0.0f;
        E8QC_CUDA(cudaEventElapsedTime(&ms, ws.scan_ev0, ws.scan_ev1));
        x->prof.scan_launches += 1;
        x->prof.scan_ms += ms;
        x->prof.candidates += cnt[0];
        x->prof.list_vectors += cnt[1];
        x->prof.list_once += cnt[2];
        // algorithmic bytes of the scan kernel: per vector of a probed list
        // (once per call) its codes + (g1, h3) (batched), or its int8 proxy
        // row + (g1, h3) plus 4 bytes of proxy distance written per (query,
        // vector) pair (precision); item_bytes counts every work item's read
        const uint64_t per_vec = mode == E8QC_MODE_PRECISION ? static_cast<uint64_t>(x->pd) + 8
                                                             : static_cast<uint64_t>(x->bits) * x->pd / 8 + 8;
        const uint64_t writes = mode == E8QC_MODE_PRECISION ? cnt[0] * 2 : 0;  // fp16 proxy distances
        x->prof.algo_bytes += cnt[2] * per_vec + writes;
        x->prof.item_bytes += cnt[1] * per_vec + writes;
        x->prof.queries += nq;
        if (mode == E8QC_MODE_PRECISION) {
            // select + rescore: every proxy distance read once, then per query
            // C candidates' codes + (g1, h3) + id
            float fms = 0.0f;
            E8QC_CUDA(cudaEventElapsedTime(&fms, ws.final_ev0, ws.final_ev1));
            x->prof.final_launches += 1;
            x->prof.final_ms += fms;
            float pms = 0.0f;
            E8QC_CUDA(cudaEventElapsedTime(&pms, ws.prep_ev0, ws.prep_ev1));
            x->prof.prep_ms += pms;
            x->prof.final_bytes += cnt[0] * 2 + static_cast<uint64_t>(nq) *
                                                    static_cast<uint64_t>(precision_candidates(static_cast<int>(k))) *
                                                    (static_cast<uint64_t>(x->bits) * x->pd / 8 + 12);
        }
    }
    return static_cast<uint64_t>(launches);
}

}  // namespace

namespace e8qc {
// ---- plans and the serving loop (plan.cpp, server.cpp) ----

namespace {

class E8qTarget final : public SearchTarget {
   public:
    explicit E8qTarget(e8qc_index* x) : x_(x) {
        require_built(x, "serve");
        dim = x->dim;
        nlist = x->nlist;
        device = x->device;
    }
    void check_mode(int mode) const override {
        if (mode != E8QC_MODE_BATCHED && mode != E8QC_MODE_PRECISION)
            fail(E8QC_EINVAL, "plans and servers cover E8QC_MODE_BATCHED and E8QC_MODE_PRECISION");
    }
    // The precision proxy plane, under the index lock, synchronised.
    void prepare(int mode) override {
        require_built(x_, "serve");
        std::lock_guard<std::mutex> lock(x_->mu);
        DeviceGuard g(x_->device);
        if (mode == E8QC_MODE_PRECISION && x_->view.proxy == nullptr) {
            ensure_precision_planes(x_, nullptr);
            E8QC_CUDA(cudaStreamSynchronize(nullptr));
        }
    }
    // Workspace buffers plus the caller's query / k / nprobe / result buffers.
    size_t bytes(int mode, size_t nq, size_t k_max, size_t np_max) const override {
        const size_t np = std::min(np_max, x_->nlist), nl = x_->nlist, pd = x_->pd;
        const size_t npairs = nq * np;
        const size_t align = mode == E8QC_MODE_PRECISION ? 8 : 1;
        const size_t pslots = npairs + (align - 1) * nl;
        size_t b = nq * (x_->dim * 4 + pd * 4 + k_max * 8 + 8);  // queries, rotated queries, results, k/nprobe
        b += nq * nl * 8 + nq * 4;                                // route keys, norms
        b += npairs * 12 + pslots * 8 + nl * 12;                  // probes, d2, positions; pair rows; list counters
        b += (npairs / 64 + nl + 1) * 16 + 32;                    // work items
        if (mode == E8QC_MODE_PRECISION) {
            const size_t rows_q = max_tiles_for(x_, np) * 32;  // proxy rows one query can need
            b += nq * (pd + 12) + nl * 8;                      // int8 queries, scales, row bases
            b += precision_row_scratch(nq, rows_q);            // proxy rows of one chunk
            b += ((pslots + 7) / 8 * 8 + 128) * pd;  // gathered int8 query rows
        } else {
            b += npairs * k_max * 8;  // per-pair partial top-k
        }
        return b;
    }
    // Kernel wait timeouts land in ws's error word. apply_tuned: take the
    // autotuned setting of this batch shape (else ws's own setting is used,
    // as a captured plan fixes it).
    uint64_t enqueue(Workspace& ws, int mode, const float* q_dev, size_t nq, const uint32_t* k_dev,
                     const uint32_t* np_dev, size_t k_max, size_t np_max, uint32_t* ids_dev, float* d_dev,
                     cudaStream_t s, bool apply_tuned) override {
        const size_t np = std::min(np_max, x_->nlist);
        ws.ensure_queries(nq, x_->pd);
        ws.ensure_err();
        float* rq = ws.rq.as<float>();
        if (apply_tuned) apply_tuning(x_, ws, mode, nq, np);
        uint64_t launches = launch_rotate(x_->view, q_dev, static_cast<int>(nq), rq, s);
        if (mode == E8QC_MODE_PRECISION)
            launches += precision_search(x_->view, ws, rq, nq, k_dev, np_dev, k_max, np, k_max, ids_dev, d_dev,
                                         max_tiles_for(x_, np) * 32, s);
        else
            launches += batched_search(x_->view, ws, rq, nq, k_dev, np_dev, k_max, np, k_max, ids_dev, d_dev,
                                       max_tiles_for(x_, np), s);
        return launches;
    }
    void autotune(Workspace& ws, int mode, size_t nq, size_t k, size_t np, cudaStream_t s, int* sched,
                  int* stages) override {
        const TuneResult r = autotune_run(x_, ws, mode, nq, k, np, s);
        *sched = r.sched;
        *stages = r.stages;
    }
    void stored_tuning(Workspace& ws, int mode, size_t nq, size_t np) override { apply_tuning(x_, ws, mode, nq, np); }

   private:
    e8qc_index* x_;
};

}  // namespace

std::shared_ptr<SearchTarget> e8q_target(e8qc_index* x) { return std::make_shared<E8qTarget>(x); }

// Read-only view of a built index for the no-allocation plain search
// (noalloc.cu). Throws like every entry point when the index is not built.
// The returned lock holds the index mutex: the caller keeps it until its
// kernels have finished, so a concurrent build or load cannot free or replace
// the buffers the view points at.
std::unique_lock<std::mutex> plain_context(e8qc_index* x, size_t nprobe, DevIndex* view, int* device,
                                           size_t* nlist, size_t* dim, size_t* max_tiles) {
    if (x == nullptr) fail(E8QC_EINVAL, "null index");
    std::unique_lock<std::mutex> lock(x->mu);
    require_built(x, "search");
    *view = x->view;
    *device = x->device;
    *nlist = x->nlist;
    *dim = x->dim;
    *max_tiles = max_tiles_for(x, nprobe);
    return lock;
}
}  // namespace e8qc

// ---------------------------------------------------------------------------
extern "C" {

const char* e8qc_last_error(void) { return last_error(); }
int e8qc_version(void) { return 10000; }

int e8qc_branch_levels(int bits, int branch, double* out) {
    return guarded([&] {
        if (bits < 1 || bits > kMaxBits) fail(E8QC_EINVAL, "bits must be in [1, 13]");
        if (branch != 0 && branch != 1) fail(E8QC_EINVAL, "branch must be 0 or 1");
        if (out == nullptr) fail(E8QC_EINVAL, "null output");
        const std::vector<double> l = branch_levels(bits, branch);
        std::memcpy(out, l.data(), l.size() * sizeof(double));
    });
}

int e8qc_fixed_scale(int bits, double* out) {
    return guarded([&] {
        if (out == nullptr) fail(E8QC_EINVAL, "null output");
        *out = fixed_scale(bits);
    });
}

int e8qc_encode(int device, int bits, const float* unit, size_t n, size_t padded_dim,
                uint16_t* digits, uint8_t* branch, void* stream) {
    return guarded([&] {
        if (bits < 1 || bits > kMaxBits) fail(E8QC_EINVAL, "EncodeVectorAtScale: bits must be in [1, 13]");
        if (padded_dim == 0 || padded_dim % 8 != 0) fail(E8QC_EINVAL, "padded_dim must be a positive multiple of 8");
        if (n == 0) return;
        if (!unit || !digits || !branch) fail(E8QC_EINVAL, "null buffer");
        DeviceGuard g(device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const DevEncTables& et = enc_tables_device(device, bits);
        const size_t B = padded_dim / 8;
        DevBuf tu, td, tb;
        const float* ud = stage_in(unit, n * padded_dim, tu, s);
        const bool dd = is_device_ptr(digits), bd = is_device_ptr(branch);
        uint16_t* dg = digits;
        uint8_t* br = branch;
        if (!dd) { td.alloc(n * B * 8 * sizeof(uint16_t)); dg = td.as<uint16_t>(); }
        if (!bd) { tb.alloc(n * B); br = tb.as<uint8_t>(); }
        const double srd = fixed_scale(bits) * std::sqrt(static_cast<double>(padded_dim));
        launch_encode(et, ud, n, static_cast<int>(padded_dim), srd, dg, br, s);
        if (!dd) E8QC_CUDA(cudaMemcpyAsync(digits, dg, n * B * 8 * sizeof(uint16_t), cudaMemcpyDeviceToHost, s));
        if (!bd) E8QC_CUDA(cudaMemcpyAsync(branch, br, n * B, cudaMemcpyDeviceToHost, s));
        E8QC_CUDA(cudaStreamSynchronize(s));
    });
}

int e8qc_rotate(int device, size_t dim, uint64_t seed, const float* src, size_t n, float* dst,
                void* stream) {
    return guarded([&] {
        if (dim == 0) fail(E8QC_EINVAL, "dim must be positive");
        if (n == 0) return;
        if (!src || !dst) fail(E8QC_EINVAL, "null buffer");
        DeviceGuard g(device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t pd = (dim + 63) / 64 * 64;
        const std::vector<uint8_t> sg = rotator_signs(dim, seed);
        DevBuf sd, ts, tdst;
        sd.alloc(sg.size());
        E8QC_CUDA(cudaMemcpyAsync(sd.p, sg.data(), sg.size(), cudaMemcpyHostToDevice, s));
        const float* in = stage_in(src, n * dim, ts, s);
        const bool dd = is_device_ptr(dst);
        float* out = dst;
        if (!dd) { tdst.alloc(n * pd * sizeof(float)); out = tdst.as<float>(); }
        launch_rotate_raw(sd.as<uint8_t>(), static_cast<int>(dim), static_cast<int>(pd), in,
                          static_cast<int>(n), out, nullptr, s);
        if (!dd) E8QC_CUDA(cudaMemcpyAsync(dst, out, n * pd * sizeof(float), cudaMemcpyDeviceToHost, s));
        E8QC_CUDA(cudaStreamSynchronize(s));
    });
}

}  // extern "C"

namespace {

// The device view of an index whose buffers are in place (build, load); a new
// layout invalidates the precision plane.
void set_view(e8qc_index* x) {
    {
        // a captured graph points into the old view's buffers
        std::lock_guard<std::mutex> gl(x->gmu);
        x->gplan.reset();
        x->glast = e8qc_index::GraphKey{};
        x->gkey = e8qc_index::GraphKey{};
    }
    DevIndex& v = x->view;
    v.dim = static_cast<int>(x->dim);
    v.pd = static_cast<int>(x->pd);
    v.B = x->B;
    v.bits = x->bits;
    v.nlist = static_cast<int>(x->nlist);
    v.nch = x->nch;
    v.ntiles = static_cast<int>(x->ntiles);
    v.signs = x->signs.as<uint8_t>();
    v.mean_rot = x->mean_rot.as<float>();
    v.cen = x->cen.as<float>();
    v.cn2 = x->cn2.as<float>();
    v.tile_begin = x->tile_begin_d.as<uint32_t>();
    v.list_len = x->list_len_d.as<uint32_t>();
    v.codes = static_cast<const uint4*>(x->codes.p);
    v.g1 = x->g1.as<float>();
    v.h3 = x->h3.as<float>();
    v.ids = x->ids.as<uint32_t>();
    v.tab = x->tab.as<float>();
    v.list_order = x->list_order.as<uint32_t>();
    v.list_of_tile = x->list_of_tile.as<uint32_t>();
    x->proxy.release();
    x->vcodes.release();
    x->rowa.release();
    x->banks_d.release();
    v.proxy = nullptr;
    v.vcodes = nullptr;
}

// The host list layout and the small device tables every index carries:
// tiles, list lengths, tile -> list, work-queue orders and the level table.
void install_lists(e8qc_index* x, const std::vector<uint64_t>& counts, cudaStream_t s) {
    const size_t nlist = x->nlist;
    x->list_begin.assign(nlist + 1, 0);
    x->tile_begin.assign(nlist + 1, 0);
    for (size_t c = 0; c < nlist; ++c) {
        x->list_begin[c + 1] = x->list_begin[c] + counts[c];
        x->tile_begin[c + 1] = x->tile_begin[c] + static_cast<uint32_t>((counts[c] + 31) / 32);
    }
    x->ntiles = x->tile_begin[nlist];
    std::vector<uint32_t> t(nlist), list_len(nlist), list_of_tile(std::max<size_t>(1, x->ntiles), 0);
    for (size_t c = 0; c < nlist; ++c) {
        t[c] = x->tile_begin[c + 1] - x->tile_begin[c];
        list_len[c] = static_cast<uint32_t>(counts[c]);
        for (uint32_t tl = x->tile_begin[c]; tl < x->tile_begin[c + 1]; ++tl) list_of_tile[tl] = static_cast<uint32_t>(c);
    }
    std::sort(t.begin(), t.end(), std::greater<uint32_t>());
    x->sorted_tiles_prefix.assign(nlist + 1, 0);
    for (size_t c = 0; c < nlist; ++c) x->sorted_tiles_prefix[c + 1] = x->sorted_tiles_prefix[c] + t[c];
    x->tile_begin_d.upload(x->tile_begin.data(), x->tile_begin.size() * 4, s);
    x->list_len_d.upload(list_len.data(), list_len.size() * 4, s);
    x->list_of_tile.upload(list_of_tile.data(), list_of_tile.size() * 4, s);
    x->list_begin_d.upload(x->list_begin.data(), x->list_begin.size() * 8, s);
    std::vector<uint32_t> order(2 * nlist);
    for (size_t c = 0; c < nlist; ++c) order[c] = order[nlist + c] = static_cast<uint32_t>(c);
    std::stable_sort(order.begin(), order.begin() + nlist, [&](uint32_t a, uint32_t b) { return counts[a] > counts[b]; });
    x->list_order.upload(order.data(), order.size() * 4, s);
    const int q = 1 << x->bits;
    std::vector<float> tab(2 * static_cast<size_t>(q));
    const double rd = std::sqrt(static_cast<double>(x->pd));
    for (int br = 0; br < 2; ++br) {
        const std::vector<double> lev = branch_levels(x->bits, br);
        for (int d = 0; d < q; ++d) tab[br * q + d] = static_cast<float>(lev[d] / rd);
    }
    x->tab.upload(tab.data(), tab.size() * 4, s);
}

size_t sign_bytes(size_t dim) { return rotator_signs(dim, 0).size(); }

// Branch-averaged level mean of each top-bit class (ScanClassMeans,
// src/quantization/e8q_codec.cpp:511-524): the basis the reference's scan
// banks price each digit at.
void scan_class_means(int bits, double w_cls[2]) {
    const std::vector<double> l0 = branch_levels(bits, 0), l1 = branch_levels(bits, 1);
    const int cvals = 1 << (bits - 1);
    for (int t2 = 0; t2 < 2; ++t2) {
        double s0 = 0.0, s1 = 0.0;
        for (int lo = 0; lo < cvals; ++lo) {
            s0 += l0[static_cast<size_t>((t2 << (bits - 1)) | lo)];
            s1 += l1[static_cast<size_t>((t2 << (bits - 1)) | lo)];
        }
        w_cls[t2] = 0.5 * (s0 / cvals + s1 / cvals);
    }
}

}  // namespace

extern "C" {

int e8qc_e8q_load(int device, const char* path, e8qc_index** out) {
    return guarded([&] {
        if (out == nullptr) fail(E8QC_EINVAL, "null output");
        *out = nullptr;
        int ndev = 0;
        E8QC_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) fail(E8QC_EINVAL, "no such CUDA device");
        E8axParts p = read_e8ax(path, sign_bytes);
        auto x = std::make_unique<e8qc_index>();
        x->device = device;
        x->dim = p.dim;
        x->pd = p.pd;
        x->bits = p.bits;
        x->seed = 0;
        x->B = static_cast<int>(p.pd / 8);
        x->nch = p.nch;
        x->ws.device = device;
        x->n = p.n;
        x->nlist = p.nlist;
        x->prune_alpha = p.prune_alpha;
        DeviceGuard g(device);
        cudaStream_t s = nullptr;
        std::vector<uint64_t> counts(p.nlist);
        for (size_t c = 0; c < p.nlist; ++c) counts[c] = p.list_begin[c + 1] - p.list_begin[c];
        install_lists(x.get(), counts, s);
        x->ids_compact = std::move(p.ids_compact);
        x->signs.upload(p.signs.data(), p.signs.size(), s);
        x->mean_rot.upload(p.mean_rot.data(), p.mean_rot.size() * 4, s);
        x->cen.upload(p.cen_rot.data(), p.cen_rot.size() * 4, s);
        x->cn2.upload(p.cn2.data(), p.cn2.size() * 4, s);
        x->codes.upload(p.codes.data(), p.codes.size() * sizeof(uint4), s);
        x->g1.upload(p.g1.data(), p.g1.size() * 4, s);
        x->h3.upload(p.h3.data(), p.h3.size() * 4, s);
        x->ids.upload(p.slot_ids.data(), p.slot_ids.size() * 4, s);
        x->banks = std::move(p.banks);
        set_view(x.get());
        E8QC_CUDA(cudaStreamSynchronize(s));
        x->built = true;
        *out = x.release();
    });
}

int e8qc_e8q_create(int device, size_t dim, int nbits, uint64_t seed, e8qc_index** out) {
    return guarded([&] {
        if (out == nullptr) fail(E8QC_EINVAL, "null output");
        *out = nullptr;
        if (dim == 0) fail(E8QC_EINVAL, "dim must be positive");
        if (nbits < 1 || nbits > kMaxBits) fail(E8QC_EINVAL, "nbits must be in [1, 13]");
        host_alloc_point();
        int ndev = 0;
        E8QC_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) fail(E8QC_EINVAL, "no such CUDA device");
        auto x = std::make_unique<e8qc_index>();
        x->device = device;
        x->dim = dim;
        x->pd = (dim + 63) / 64 * 64;
        x->bits = nbits;
        x->seed = seed;
        x->B = static_cast<int>(x->pd / 8);
        x->nch = code_chunks(static_cast<int>(x->pd), nbits);
        x->ws.device = device;
        *out = x.release();
    });
}

int e8qc_debug_fail_host_allocs(int count) {
    return guarded([&] {
        if (count < 0) fail(E8QC_EINVAL, "count must be >= 0");
        g_fail_host_allocs.store(count);
    });
}

int e8qc_e8q_debug_inject_wait_timeout(e8qc_index* x, int searches, uint32_t wait_ms) {
    return guarded([&] {
        if (x == nullptr) fail(E8QC_EINVAL, "null index");
        if (searches < 0) fail(E8QC_EINVAL, "searches must be >= 0");
        if (searches > 0 && (wait_ms < 1 || wait_ms > 10000)) fail(E8QC_EINVAL, "wait_ms must be in [1, 10000]");
        x->inject_wait_ms.store(wait_ms);
        x->inject_waits.store(searches);
    });
}

int e8qc_e8q_destroy(e8qc_index* x) {
    return guarded([&] {
        if (x == nullptr) return;
        DeviceGuard g(x->device);
        delete x;
    });
}

int e8qc_e8q_build(e8qc_index* x, const float* data, size_t n, const float* centroids, size_t nlist,
                   const uint32_t* cluster_ids, float prune_alpha, void* stream) {
    return guarded([&] {
        if (x == nullptr) fail(E8QC_EINVAL, "null index");
        if (n == 0 || nlist == 0) fail(E8QC_EINVAL, "BuildLists: empty input");
        if (!data || !centroids || !cluster_ids) fail(E8QC_EINVAL, "null buffer");
        if (n > 0xFFFFFFFEull) fail(E8QC_EINVAL, "too many vectors for 32-bit ids");
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // cluster ids on the host for the list layout
        std::vector<uint32_t> cid_h;
        const uint32_t* cid = cluster_ids;
        if (is_device_ptr(cluster_ids)) {
            cid_h.resize(n);
            E8QC_CUDA(cudaMemcpyAsync(cid_h.data(), cluster_ids, n * 4, cudaMemcpyDeviceToHost, s));
            E8QC_CUDA(cudaStreamSynchronize(s));
            cid = cid_h.data();
        }
        std::vector<uint64_t> counts(nlist, 0);
        for (size_t i = 0; i < n; ++i) {
            if (cid[i] >= nlist) fail(E8QC_EINVAL, "cluster id out of range");
            ++counts[cid[i]];
        }
        x->built = false;
        x->n = n;
        x->nlist = nlist;
        x->prune_alpha = prune_alpha > 0.0f ? prune_alpha : 1.0f;
        x->list_begin.assign(nlist + 1, 0);
        x->tile_begin.assign(nlist + 1, 0);
        for (size_t c = 0; c < nlist; ++c) {
            x->list_begin[c + 1] = x->list_begin[c] + counts[c];
            x->tile_begin[c + 1] = x->tile_begin[c] + static_cast<uint32_t>((counts[c] + 31) / 32);
        }
        x->ntiles = x->tile_begin[nlist];
        {
            std::vector<uint32_t> t(nlist);
            for (size_t c = 0; c < nlist; ++c) t[c] = x->tile_begin[c + 1] - x->tile_begin[c];
            std::sort(t.begin(), t.end(), std::greater<uint32_t>());
            x->sorted_tiles_prefix.assign(nlist + 1, 0);
            for (size_t c = 0; c < nlist; ++c) x->sorted_tiles_prefix[c + 1] = x->sorted_tiles_prefix[c] + t[c];
        }
        // posting lists in file order (src/index/e8q_build.cpp:120-133)
        std::vector<uint32_t> row_of(x->ntiles * 32, 0xFFFFFFFFu);
        std::vector<uint32_t> list_of_tile(x->ntiles);
        std::vector<uint32_t> list_len(nlist);
        x->ids_compact.assign(n, 0);
        {
            std::vector<uint64_t> cursor(nlist, 0);
            for (size_t i = 0; i < n; ++i) {
                const uint32_t c = cid[i];
                const uint64_t r = cursor[c]++;
                row_of[static_cast<size_t>(x->tile_begin[c]) * 32 + r] = static_cast<uint32_t>(i);
                x->ids_compact[x->list_begin[c] + r] = static_cast<uint32_t>(i);
            }
            for (size_t c = 0; c < nlist; ++c) {
                list_len[c] = static_cast<uint32_t>(counts[c]);
                for (uint32_t t = x->tile_begin[c]; t < x->tile_begin[c + 1]; ++t) list_of_tile[t] = static_cast<uint32_t>(c);
            }
        }
        x->inv_pos.clear();
        const size_t pd = x->pd, dim = x->dim;
        // device state
        const std::vector<uint8_t> sg = rotator_signs(dim, x->seed);
        x->signs.upload(sg.data(), sg.size(), s);
        x->tile_begin_d.upload(x->tile_begin.data(), x->tile_begin.size() * 4, s);
        x->list_len_d.upload(list_len.data(), list_len.size() * 4, s);
        x->ids.upload(row_of.data(), row_of.size() * 4, s);
        x->list_of_tile.upload(list_of_tile.data(), list_of_tile.size() * 4, s);
        x->list_begin_d.upload(x->list_begin.data(), x->list_begin.size() * 8, s);
        {
            // batched work queue orders: longest list first (LPT), then list id order
            std::vector<uint32_t> order(2 * nlist);
            for (size_t c = 0; c < nlist; ++c) order[c] = order[nlist + c] = static_cast<uint32_t>(c);
            std::stable_sort(order.begin(), order.begin() + nlist,
                             [&](uint32_t a, uint32_t b) { return counts[a] > counts[b]; });
            x->list_order.upload(order.data(), order.size() * 4, s);
        }
        {
            // refine tables: level / sqrt(pd) as float (src/quantization/e8q_codec.cpp:933-946)
            const int q = 1 << x->bits;
            std::vector<float> tab(2 * static_cast<size_t>(q));
            const double rd = std::sqrt(static_cast<double>(pd));
            for (int br = 0; br < 2; ++br) {
                const std::vector<double> lev = branch_levels(x->bits, br);
                for (int d = 0; d < q; ++d) tab[br * q + d] = static_cast<float>(lev[d] / rd);
            }
            x->tab.upload(tab.data(), tab.size() * 4, s);
        }
        DevBuf tdata, tcen, mu;
        const float* data_d = stage_in(data, n * dim, tdata, s);
        const float* cen_raw = stage_in(centroids, nlist * dim, tcen, s);
        mu.alloc(dim * sizeof(float));
        x->mean_rot.alloc(pd * sizeof(float));
        x->cen.alloc(nlist * pd * sizeof(float));
        x->cn2.alloc(nlist * sizeof(float));
        x->codes.alloc(x->ntiles * static_cast<size_t>(x->nch) * 32 * 16);
        x->g1.alloc(x->ntiles * 32 * sizeof(float));
        x->h3.alloc(x->ntiles * 32 * sizeof(float));
        x->ortho.alloc(x->ntiles * 32 * 3 * sizeof(float));
        x->banks.clear();
        E8QC_CUDA(cudaMemsetAsync(x->codes.p, 0, x->codes.bytes, s));
        // mean -> rotated mean -> centroids
        launch_mean(data_d, n, static_cast<int>(dim), mu.as<float>(), s);
        launch_rotate_raw(x->signs.as<uint8_t>(), static_cast<int>(dim), static_cast<int>(pd), mu.as<float>(), 1,
                          x->mean_rot.as<float>(), nullptr, s);
        launch_centroids(x->signs.as<uint8_t>(), static_cast<int>(dim), static_cast<int>(pd), cen_raw,
                         static_cast<int>(nlist), x->mean_rot.as<float>(), x->cen.as<float>(),
                         x->cn2.as<float>(), s);
        set_view(x);
        DevIndex& v = x->view;
        const DevEncTables& et = enc_tables_device(x->device, x->bits);
        BuildEncodeArgs a{};
        a.base = data_d;
        a.row_of = x->ids.as<uint32_t>();
        a.list_of_tile = x->list_of_tile.as<uint32_t>();
        a.ntiles = static_cast<int>(x->ntiles);
        a.srd = fixed_scale(x->bits) * std::sqrt(static_cast<double>(pd));
        a.inv_level_scale = 1.0 / std::sqrt(static_cast<double>(pd));
        scan_class_means(x->bits, a.w_cls);
        a.ortho = x->ortho.as<float>();
        launch_build_encode(v, et, a, static_cast<uint4*>(x->codes.p), x->g1.as<float>(), x->h3.as<float>(), s);
        E8QC_CUDA(cudaStreamSynchronize(s));
        x->built = true;
    });
}

int e8qc_e8q_search(e8qc_index* x, const float* queries, size_t nq, size_t k, size_t nprobe, int mode,
                    uint32_t* out_ids, float* out_dists, e8qc_stats* stats, void* stream) {
    return guarded([&] {
        require_built(x, "search");
        if (k == 0) fail(E8QC_EINVAL, "k must be positive");
        if (k > static_cast<size_t>(kMaxK)) fail(E8QC_EINVAL, "k must be <= 128");
        if (nprobe == 0) fail(E8QC_EINVAL, "nprobe must be positive");
        if (mode != E8QC_MODE_PLAIN && mode != E8QC_MODE_BATCHED && mode != E8QC_MODE_PRECISION &&
            mode != E8QC_MODE_PRUNED)
            fail(E8QC_EINVAL, "unknown search mode");
        if (nq == 0) return;
        if (!queries || !out_ids) fail(E8QC_EINVAL, "null buffer");
        // a repeated large batch shape of a grouped mode replays a captured graph
        std::shared_ptr<e8qc_plan> plan;
        // (host-resident queries only: device-resident ones would add a copy
        // into the plan's staging, and the direct path keeps the GPU as busy)
        if (mode != E8QC_MODE_PLAIN && mode != E8QC_MODE_PRUNED && nq >= kGraphMinQueries && !x->profiling &&
            !is_device_ptr(queries)) {
            const e8qc_index::GraphKey key{mode, nq, k, std::min(nprobe, x->nlist)};
            bool create = false;
            {
                std::lock_guard<std::mutex> gl(x->gmu);
                if (x->gplan && x->gkey == key) plan = x->gplan;
                else if (x->glast == key) create = true;
                else x->glast = key;
            }
            if (create) {
                try {
                    plan = std::shared_ptr<e8qc_plan>(plan_make(e8q_target(x), mode, nq, k, key.np, false, true),
                                                      plan_free);
                    std::lock_guard<std::mutex> gl(x->gmu);
                    x->gplan = plan;
                    x->gkey = key;
                } catch (const Error&) {
                    plan.reset();  // e.g. no memory for a second workspace: the direct path below
                }
            }
        }
        std::lock_guard<std::mutex> lock(x->mu);
        if (plan) {
            // a build or load between the lookup above and taking the index
            // mutex resets the cached plan (its graph points at freed
            // buffers): replay only the plan that is still current
            std::lock_guard<std::mutex> gl(x->gmu);
            if (x->gplan != plan) plan.reset();
        }
        DeviceGuard g(x->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const size_t np = std::min(nprobe, x->nlist);
        if (plan) {
            const std::vector<uint32_t> kh(nq, static_cast<uint32_t>(k)), nph(nq, static_cast<uint32_t>(np));
            cudaEvent_t ge[2] = {nullptr, nullptr};
            if (stats) {
                std::memset(stats, 0, sizeof(*stats));
                for (auto& e : ge) E8QC_CUDA(cudaEventCreate(&e));
                E8QC_CUDA(cudaEventRecord(ge[0], s));
            }
            plan_enqueue(plan.get(), queries, nq, kh.data(), nph.data(), out_ids, out_dists, s);
            if (stats) E8QC_CUDA(cudaEventRecord(ge[1], s));
            plan_check(plan.get(), s);
            if (stats) {
                // a replayed graph reports its whole device time (with the
                // staging copies) as scan_us
                float t = 0;
                E8QC_CUDA(cudaEventElapsedTime(&t, ge[0], ge[1]));
                stats->scan_us = t * 1000.0;
                stats->launches = plan_kernels(plan.get());
                for (auto& e : ge) cudaEventDestroy(e);
            }
            return;
        }
        if (stats) std::memset(stats, 0, sizeof(*stats));
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
        if (stats)
            for (auto& e : ev) E8QC_CUDA(cudaEventCreate(&e));
        // host-buffer staging lives in the workspace (grown, never freed per call:
        // cudaFree would synchronise the device on every search)
        DevBuf& tq = x->ws.stage_q;
        DevBuf& tids = x->ws.stage_ids;
        DevBuf& tds = x->ws.stage_d;
        const float* qd = stage_in(queries, nq * x->dim, tq, s);
        const bool ids_dev = is_device_ptr(out_ids);
        const bool d_dev = out_dists != nullptr && is_device_ptr(out_dists);
        uint32_t* ids_d = out_ids;
        float* d_d = out_dists;
        if (!ids_dev) { tids.ensure(nq * k * 4); ids_d = tids.as<uint32_t>(); }
        if (!d_dev) { tds.ensure(nq * k * 4); d_d = tds.as<float>(); }
        x->ws.ensure_queries(nq, x->pd);
        float* rq = x->ws.rq.as<float>();
        uint64_t launches = 0;
        if (stats) E8QC_CUDA(cudaEventRecord(ev[0], s));
        launches += launch_rotate(x->view, qd, static_cast<int>(nq), rq, s);
        if (stats) E8QC_CUDA(cudaEventRecord(ev[1], s));
        if (mode == E8QC_MODE_PLAIN) {
            plain_search(x, rq, nq, k, np, ids_d, d_d, stats, s);
        } else if (mode == E8QC_MODE_PRUNED) {
            pruned_search(x, rq, nq, k, np, ids_d, d_d, stats, s);
        } else {
            launches += grouped_search(x, mode, rq, nq, nullptr, nullptr, k, np, ids_d, d_d, s);
        }
        if (stats) E8QC_CUDA(cudaEventRecord(ev[2], s));
        if (!ids_dev) E8QC_CUDA(cudaMemcpyAsync(out_ids, ids_d, nq * k * 4, cudaMemcpyDeviceToHost, s));
        if (out_dists && !d_dev) E8QC_CUDA(cudaMemcpyAsync(out_dists, d_d, nq * k * 4, cudaMemcpyDeviceToHost, s));
        x->ws.check_error(s);
        if (stats) {
            float a = 0, b = 0;
            E8QC_CUDA(cudaEventElapsedTime(&a, ev[0], ev[1]));
            E8QC_CUDA(cudaEventElapsedTime(&b, ev[1], ev[2]));
            stats->rotate_us = a * 1000.0;
            stats->scan_us = b * 1000.0;
            stats->launches += launches;
            // every candidate of every probed list is scored exactly
            uint64_t cand = 0;
            (void)cand;
            for (auto& e : ev) cudaEventDestroy(e);
        }
    });
}

int e8qc_e8q_search_ragged(e8qc_index* x, const float* queries, size_t nq, const uint32_t* k,
                           const uint32_t* nprobe, size_t k_max, uint32_t* out_ids, float* out_dists,
                           e8qc_stats* stats, void* stream) {
    return e8qc_e8q_search_ragged_mode(x, queries, nq, k, nprobe, k_max, E8QC_MODE_BATCHED, out_ids, out_dists,
                                       stats, stream);
}

int e8qc_e8q_search_ragged_mode(e8qc_index* x, const float* queries, size_t nq, const uint32_t* k,
                                const uint32_t* nprobe, size_t k_max, int mode, uint32_t* out_ids,
                                float* out_dists, e8qc_stats* stats, void* stream) {
    return guarded([&] {
        require_built(x, "search");
        if (mode != E8QC_MODE_BATCHED && mode != E8QC_MODE_PRECISION)
            fail(E8QC_EINVAL, "ragged search runs the batched or precision mode");
        if (k_max == 0 || k_max > static_cast<size_t>(kMaxK)) fail(E8QC_EINVAL, "k_max must be in [1, 128]");
        if (nq == 0) return;
        if (!queries || !k || !nprobe || !out_ids) fail(E8QC_EINVAL, "null buffer");
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (stats) std::memset(stats, 0, sizeof(*stats));
        // per-query parameters on the host for validation and bounds
        std::vector<uint32_t> kh(nq), nph(nq);
        if (is_device_ptr(k)) E8QC_CUDA(cudaMemcpy(kh.data(), k, nq * 4, cudaMemcpyDeviceToHost));
        else std::memcpy(kh.data(), k, nq * 4);
        if (is_device_ptr(nprobe)) E8QC_CUDA(cudaMemcpy(nph.data(), nprobe, nq * 4, cudaMemcpyDeviceToHost));
        else std::memcpy(nph.data(), nprobe, nq * 4);
        size_t np_max = 0;
        for (size_t i = 0; i < nq; ++i) {
            if (kh[i] == 0 || kh[i] > k_max) fail(E8QC_EINVAL, "k must be in [1, k_max]");
            if (nph[i] == 0) fail(E8QC_EINVAL, "nprobe must be positive");
            nph[i] = static_cast<uint32_t>(std::min<size_t>(nph[i], x->nlist));
            np_max = std::max<size_t>(np_max, nph[i]);
        }
        DevBuf& tq = x->ws.stage_q;
        DevBuf& tk = x->ws.stage_k;
        DevBuf& tnp = x->ws.stage_np;
        DevBuf& tids = x->ws.stage_ids;
        DevBuf& tds = x->ws.stage_d;
        const float* qd = stage_in(queries, nq * x->dim, tq, s);
        tk.ensure(nq * 4);
        tnp.ensure(nq * 4);
        E8QC_CUDA(cudaMemcpyAsync(tk.p, kh.data(), nq * 4, cudaMemcpyHostToDevice, s));
        E8QC_CUDA(cudaMemcpyAsync(tnp.p, nph.data(), nq * 4, cudaMemcpyHostToDevice, s));
        const bool ids_dev = is_device_ptr(out_ids);
        const bool d_dev = out_dists != nullptr && is_device_ptr(out_dists);
        uint32_t* ids_d = out_ids;
        float* d_d = out_dists;
        if (!ids_dev) { tids.ensure(nq * k_max * 4); ids_d = tids.as<uint32_t>(); }
        if (!d_dev) { tds.ensure(nq * k_max * 4); d_d = tds.as<float>(); }
        x->ws.ensure_queries(nq, x->pd);
        float* rq = x->ws.rq.as<float>();
        uint64_t launches = launch_rotate(x->view, qd, static_cast<int>(nq), rq, s);
        launches += grouped_search(x, mode, rq, nq, tk.as<uint32_t>(), tnp.as<uint32_t>(), k_max, np_max, ids_d,
                                   d_d, s);
        if (!ids_dev) E8QC_CUDA(cudaMemcpyAsync(out_ids, ids_d, nq * k_max * 4, cudaMemcpyDeviceToHost, s));
        if (out_dists && !d_dev) E8QC_CUDA(cudaMemcpyAsync(out_dists, d_d, nq * k_max * 4, cudaMemcpyDeviceToHost, s));
        x->ws.check_error(s);
        if (stats) stats->launches = launches;
    });
}

int e8qc_e8q_estimate(e8qc_index* x, const float* query, uint32_t id, float* out) {
    return guarded([&] {
        require_built(x, "estimate");
        if (!query || !out) fail(E8QC_EINVAL, "null buffer");
        std::lock_guard<std::mutex> lock(x->mu);
        if (x->inv_pos.size() != x->n) {
            x->inv_pos.assign(x->n, 0xFFFFFFFFu);
            for (size_t i = 0; i < x->n; ++i) x->inv_pos[x->ids_compact[i]] = static_cast<uint32_t>(i);
        }
        if (id >= x->n || x->inv_pos[id] == 0xFFFFFFFFu) fail(E8QC_ERANGE, "Estimate: id out of range");
        const uint64_t pos = x->inv_pos[id];
        const size_t c = static_cast<size_t>(
            std::upper_bound(x->list_begin.begin() + 1, x->list_begin.end(), pos) - x->list_begin.begin() - 1);
        const uint32_t slot = x->tile_begin[c] * 32 + static_cast<uint32_t>(pos - x->list_begin[c]);
        DeviceGuard g(x->device);
        cudaStream_t s = nullptr;
        DevBuf tq, out_d;
        const float* qd = stage_in(query, x->dim, tq, s);
        x->ws.ensure_queries(1, x->pd);
        launch_rotate(x->view, qd, 1, x->ws.rq.as<float>(), s);
        out_d.alloc(4);
        launch_estimate(x->view, x->ws.rq.as<float>(), static_cast<int>(c), slot, out_d.as<float>(), s);
        float r = 0.0f;
        E8QC_CUDA(cudaMemcpy(&r, out_d.p, 4, cudaMemcpyDeviceToHost));
        *out = r;
    });
}

int e8qc_e8q_probe_bound_w(e8qc_index* x, const float* queries, size_t nq, const float* base_rows,
                           const uint32_t* qidx, const uint32_t* ids, size_t m, double* out) {
    return guarded([&] {
        require_built(x, "probe_bound_w");
        if (m == 0) return;
        if (!queries || !base_rows || !qidx || !ids || !out) fail(E8QC_EINVAL, "null buffer");
        std::lock_guard<std::mutex> lock(x->mu);
        if (x->inv_pos.size() != x->n) {
            x->inv_pos.assign(x->n, 0xFFFFFFFFu);
            for (size_t i = 0; i < x->n; ++i) x->inv_pos[x->ids_compact[i]] = static_cast<uint32_t>(i);
        }
        DeviceGuard g(x->device);
        cudaStream_t s = nullptr;
        // per pair: the stored vector's slot and list (UINT32_MAX: NaN, as the
        // reference's binding for a query or id out of range)
        std::vector<uint32_t> qi(m), ids_h(m), slot(m, 0xFFFFFFFFu), list(m, 0);
        E8QC_CUDA(cudaMemcpy(qi.data(), qidx, m * 4, cudaMemcpyDefault));
        E8QC_CUDA(cudaMemcpy(ids_h.data(), ids, m * 4, cudaMemcpyDefault));
        for (size_t i = 0; i < m; ++i) {
            const uint32_t id = ids_h[i];
            if (qi[i] >= nq || id >= x->n || x->inv_pos[id] == 0xFFFFFFFFu) {
                qi[i] = 0;
                continue;
            }
            const uint64_t pos = x->inv_pos[id];
            const size_t c = static_cast<size_t>(
                std::upper_bound(x->list_begin.begin() + 1, x->list_begin.end(), pos) - x->list_begin.begin() - 1);
            slot[i] = x->tile_begin[c] * 32 + static_cast<uint32_t>(pos - x->list_begin[c]);
            list[i] = static_cast<uint32_t>(c);
        }
        // levels / sqrt(Dpad) of both branches and the scan basis (class means,
        // zero for dim 7 at 1 bit), in double
        const int q = 1 << x->bits;
        const double rd = std::sqrt(static_cast<double>(x->pd));
        std::vector<double> tabs(2 * static_cast<size_t>(q) + 16);
        for (int br = 0; br < 2; ++br) {
            const std::vector<double> lev = branch_levels(x->bits, br);
            for (int d = 0; d < q; ++d) tabs[static_cast<size_t>(br) * q + d] = lev[d] / rd;
        }
        double w_cls[2];
        scan_class_means(x->bits, w_cls);
        for (int d = 0; d < 8; ++d) {
            tabs[2 * q + 2 * d] = (x->bits == 1 && d == 7) ? 0.0 : w_cls[0];
            tabs[2 * q + 2 * d + 1] = (x->bits == 1 && d == 7) ? 0.0 : w_cls[1];
        }
        DevBuf tq, tb, rqd, rxd, meta, tabd, outd;
        const float* qd = stage_in(queries, nq * x->dim, tq, s);
        const float* bd = stage_in(base_rows, m * x->dim, tb, s);
        rqd.alloc(std::max<size_t>(nq, 1) * x->pd * 4);
        rxd.alloc(m * x->pd * 4);
        if (nq > 0) launch_rotate(x->view, qd, static_cast<int>(nq), rqd.as<float>(), s);
        launch_rotate(x->view, bd, static_cast<int>(m), rxd.as<float>(), s);
        meta.alloc(m * 12);
        uint32_t* md = meta.as<uint32_t>();
        E8QC_CUDA(cudaMemcpyAsync(md, qi.data(), m * 4, cudaMemcpyHostToDevice, s));
        E8QC_CUDA(cudaMemcpyAsync(md + m, slot.data(), m * 4, cudaMemcpyHostToDevice, s));
        E8QC_CUDA(cudaMemcpyAsync(md + 2 * m, list.data(), m * 4, cudaMemcpyHostToDevice, s));
        tabd.alloc(tabs.size() * 8);
        E8QC_CUDA(cudaMemcpyAsync(tabd.p, tabs.data(), tabs.size() * 8, cudaMemcpyHostToDevice, s));
        outd.alloc(m * 8);
        launch_probe_bound(x->view, rqd.as<float>(), rxd.as<float>(), md, md + m, md + 2 * m, tabd.as<double>(),
                           tabd.as<double>() + 2 * q, static_cast<int>(m), static_cast<int>(x->dim),
                           outd.as<double>(), s);
        E8QC_CUDA(cudaMemcpyAsync(out, outd.p, m * 8, cudaMemcpyDefault, s));
        E8QC_CUDA(cudaStreamSynchronize(s));
    });
}

int e8qc_e8q_set_disable_prune(e8qc_index* x, int on) {
    return guarded([&] {
        require_built(x, "set_disable_prune");
        x->disable_prune = on != 0;
    });
}

int e8qc_e8q_set_prune_alpha(e8qc_index* x, float alpha) {
    return guarded([&] {
        require_built(x, "set_prune_alpha");
        if (!(alpha > 0.0f)) fail(E8QC_EINVAL, "prune_alpha must be positive");
        x->prune_alpha = alpha;
    });
}

int e8qc_e8q_pruned_thresholds(e8qc_index* x, float* out, size_t nq) {
    return guarded([&] {
        require_built(x, "pruned_thresholds");
        if (out == nullptr && nq > 0) fail(E8QC_EINVAL, "null buffer");
        std::lock_guard<std::mutex> lock(x->mu);
        if (nq > x->ws.pr_last_nq) fail(E8QC_EINVAL, "more thresholds asked for than the last pruned search had queries");
        if (nq == 0) return;
        DeviceGuard g(x->device);
        E8QC_CUDA(cudaMemcpy(out, x->ws.pr_thr.p, nq * 4, cudaMemcpyDeviceToHost));
    });
}

int e8qc_e8q_info(const e8qc_index* x, e8qc_info* out) {
    return guarded([&] {
        if (!x || !out) fail(E8QC_EINVAL, "null argument");
        out->dim = x->dim;
        out->padded_dim = x->pd;
        out->n = x->n;
        out->nlist = x->nlist;
        out->memory_bytes = x->memory_bytes();
        out->nbits = x->bits;
        out->device = x->device;
        out->built = x->built ? 1 : 0;
        out->disable_prune = x->disable_prune ? 1 : 0;
        out->prune_alpha = x->prune_alpha;
    });
}

int e8qc_e8q_autotune(e8qc_index* x, int mode, size_t nq, size_t k, size_t nprobe, e8qc_tuning* out) {
    return guarded([&] {
        require_built(x, "autotune");
        if (mode != E8QC_MODE_BATCHED && mode != E8QC_MODE_PRECISION)
            fail(E8QC_EINVAL, "autotune covers E8QC_MODE_BATCHED and E8QC_MODE_PRECISION");
        if (nq == 0 || k == 0 || k > static_cast<size_t>(kMaxK) || nprobe == 0)
            fail(E8QC_EINVAL, "nq, nprobe must be positive and k in [1, 128]");
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = nullptr;
        if (mode == E8QC_MODE_PRECISION) ensure_precision_planes(x, s);
        const TuneResult r = autotune_run(x, x->ws, mode, nq, k, nprobe, s);
        if (out) *out = e8qc_tuning{r.sched, r.stages, r.best_ms, r.default_ms};
    });
}

int e8qc_e8q_profile(e8qc_index* x, int enable, e8qc_profile* out) {
    return guarded([&] {
        if (x == nullptr) fail(E8QC_EINVAL, "null index");
        std::lock_guard<std::mutex> lock(x->mu);
        if (enable) {
            x->prof = e8qc_profile{};
            x->profiling = true;
        } else {
            x->profiling = false;
            if (out) *out = x->prof;
        }
    });
}

int e8qc_e8q_get_ids(const e8qc_index* x, uint32_t* out) {
    return guarded([&] {
        require_built(x, "get_ids");
        if (!out) fail(E8QC_EINVAL, "null output");
        std::memcpy(out, x->ids_compact.data(), x->n * 4);
    });
}

int e8qc_e8q_save(const e8qc_index* xc, const char* path) {
    return guarded([&] {
        require_built(xc, "save");
        if (path == nullptr) fail(E8QC_EINVAL, "null path");
        e8qc_index* x = const_cast<e8qc_index*>(xc);
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = nullptr;
        const size_t n = x->n, B = static_cast<size_t>(x->B), pd = x->pd, nlist = x->nlist;
        if (x->ortho.bytes == 0 && x->banks.empty()) fail(E8QC_ESTATE, "index holds no scan banks to save");
        // codes in compact order, then the per-slot arrays mapped to it
        std::vector<uint16_t> digits(n * B * 8);
        std::vector<uint8_t> branch(n * B);
        {
            DevBuf dd, bd;
            dd.alloc(std::max<size_t>(1, n * B * 8 * 2));
            bd.alloc(std::max<size_t>(1, n * B));
            launch_decode(x->view, static_cast<int>(x->ntiles), x->list_of_tile.as<uint32_t>(),
                          x->list_begin_d.as<uint64_t>(), dd.as<uint16_t>(), bd.as<uint8_t>(), s);
            E8QC_CUDA(cudaStreamSynchronize(s));
            if (n) {
                E8QC_CUDA(cudaMemcpy(digits.data(), dd.p, n * B * 8 * 2, cudaMemcpyDeviceToHost));
                E8QC_CUDA(cudaMemcpy(branch.data(), bd.p, n * B, cudaMemcpyDeviceToHost));
            }
        }
        const size_t slots = x->ntiles * 32;
        std::vector<float> g1s(slots), h3s(slots), os(x->ortho.bytes ? slots * 3 : 0);
        E8QC_CUDA(cudaMemcpy(g1s.data(), x->g1.p, slots * 4, cudaMemcpyDeviceToHost));
        E8QC_CUDA(cudaMemcpy(h3s.data(), x->h3.p, slots * 4, cudaMemcpyDeviceToHost));
        if (!os.empty()) E8QC_CUDA(cudaMemcpy(os.data(), x->ortho.p, slots * 12, cudaMemcpyDeviceToHost));
        std::vector<float> g1(n), h3(n), ortho(os.empty() ? 0 : n * 3);
        for (size_t c = 0; c < nlist; ++c)
            for (uint64_t p = x->list_begin[c]; p < x->list_begin[c + 1]; ++p) {
                const size_t slot = static_cast<size_t>(x->tile_begin[c]) * 32 + (p - x->list_begin[c]);
                g1[p] = g1s[slot];
                h3[p] = h3s[slot];
                if (!os.empty())
                    for (int t = 0; t < 3; ++t) ortho[p * 3 + t] = os[slot * 3 + t];
            }
        std::vector<uint8_t> signs(sign_bytes(x->dim));
        std::vector<float> mean_rot(pd), cen(nlist * pd), cn2(nlist);
        E8QC_CUDA(cudaMemcpy(signs.data(), x->signs.p, signs.size(), cudaMemcpyDeviceToHost));
        E8QC_CUDA(cudaMemcpy(mean_rot.data(), x->mean_rot.p, pd * 4, cudaMemcpyDeviceToHost));
        E8QC_CUDA(cudaMemcpy(cen.data(), x->cen.p, nlist * pd * 4, cudaMemcpyDeviceToHost));
        E8QC_CUDA(cudaMemcpy(cn2.data(), x->cn2.p, nlist * 4, cudaMemcpyDeviceToHost));
        E8axSave w;
        w.n = n;
        w.dim = x->dim;
        w.nlist = nlist;
        w.pd = pd;
        w.bits = x->bits;
        w.prune_alpha = x->prune_alpha > 0.0f ? x->prune_alpha : 1.0f;
        w.signs = signs.data();
        w.sign_bytes = signs.size();
        w.mean_rot = mean_rot.data();
        w.cen_rot = cen.data();
        w.cn2 = cn2.data();
        w.list_begin = x->list_begin.data();
        w.ids = x->ids_compact.data();
        w.digits = digits.data();
        w.branch = branch.data();
        w.g1 = g1.data();
        w.h3 = h3.data();
        w.ortho = ortho.empty() ? nullptr : ortho.data();
        w.banks = ortho.empty() ? x->banks.data() : nullptr;
        write_e8ax(path, w);
    });
}

int e8qc_e8q_export_codes(const e8qc_index* xc, uint16_t* digits, uint8_t* branch, float* g1, float* h3) {
    return guarded([&] {
        require_built(xc, "export_codes");
        e8qc_index* x = const_cast<e8qc_index*>(xc);
        std::lock_guard<std::mutex> lock(x->mu);
        DeviceGuard g(x->device);
        cudaStream_t s = nullptr;
        const size_t n = x->n, B = static_cast<size_t>(x->B);
        if (digits || branch) {
            DevBuf dd, bd;
            dd.alloc(n * B * 8 * 2);
            bd.alloc(n * B);
            launch_decode(x->view, static_cast<int>(x->ntiles), x->list_of_tile.as<uint32_t>(),
                          x->list_begin_d.as<uint64_t>(), dd.as<uint16_t>(), bd.as<uint8_t>(), s);
            E8QC_CUDA(cudaStreamSynchronize(s));
            if (digits) E8QC_CUDA(cudaMemcpy(digits, dd.p, n * B * 8 * 2, cudaMemcpyDeviceToHost));
            if (branch) E8QC_CUDA(cudaMemcpy(branch, bd.p, n * B, cudaMemcpyDeviceToHost));
        }
        if (g1 || h3) {
            std::vector<float> a(x->ntiles * 32), b(x->ntiles * 32);
            E8QC_CUDA(cudaMemcpy(a.data(), x->g1.p, a.size() * 4, cudaMemcpyDeviceToHost));
            E8QC_CUDA(cudaMemcpy(b.data(), x->h3.p, b.size() * 4, cudaMemcpyDeviceToHost));
            for (size_t c = 0; c < x->nlist; ++c) {
                for (uint64_t p = x->list_begin[c]; p < x->list_begin[c + 1]; ++p) {
                    const size_t slot = static_cast<size_t>(x->tile_begin[c]) * 32 + (p - x->list_begin[c]);
                    if (g1) g1[p] = a[slot];
                    if (h3) h3[p] = b[slot];
                }
            }
        }
    });
}

}  // extern "C"
