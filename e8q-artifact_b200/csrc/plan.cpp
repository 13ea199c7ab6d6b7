// Captured search plans: a ragged batched / precision search of a fixed batch
// size recorded once as a CUDA graph and replayed per batch.
//
// Creation walks the batch sizes 64, 128, ... up to max_queries from the
// largest down: per size it autotunes (or takes the index's stored tuning),
// runs the sequence once to size the plan's own workspace -- the largest size
// first, so no later size reallocates anything a captured graph points at --
// then captures rotate + route + select + group + (quantize, gather) + scan +
// merge / rescore into a graph and instantiates it. A run pads the batch to
// the next captured size (zero queries with k = nprobe = 1), copies queries,
// k and nprobe in, launches the graph and copies the k_max-wide rows out.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "e8qc.h"
#include "internal.h"
#include "serve_target.h"
#include "workspace.h"

namespace e8qc {
void set_last_error(const std::string& s);
bool is_device_ptr(const void* p);
}  // namespace e8qc

using namespace e8qc;

struct e8qc_plan {
    std::shared_ptr<SearchTarget> target;
    int mode = 0, device = 0;
    size_t dim = 0, nlist = 0, max_q = 0, k_max = 0, np_max = 0;
    Workspace ws;
    cudaStream_t cs = nullptr;
    cudaEvent_t staged = nullptr;  // the last run's staging copies have been read
    DevBuf q, k, np, ids, d;
    uint32_t* hk = nullptr;  // pinned staging of k / nprobe (padded to the captured size)
    uint32_t* hnp = nullptr;
    struct Graph {
        size_t nq;
        cudaGraphExec_t exec;
        int sched, stages;
    };
    std::vector<Graph> graphs;  // ascending nq
    uint64_t kernels = 0;       // launched by one run of the largest graph
    ~e8qc_plan() {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        if (staged) cudaEventDestroy(staged);
        if (cs) cudaStreamDestroy(cs);
        if (hk) cudaFreeHost(hk);
        if (hnp) cudaFreeHost(hnp);
    }
};

namespace e8qc {

// Enqueue one batch (no host synchronisation): k / nprobe are host arrays of
// nq entries; queries, out_ids and out_dists may be host or device pointers
// (rows of out_* are k_max wide; out_dists may be NULL).
void plan_enqueue(e8qc_plan* P, const float* queries, size_t nq, const uint32_t* k, const uint32_t* nprobe,
                  uint32_t* out_ids, float* out_dists, cudaStream_t s) {
    if (nq == 0) return;
    if (nq > P->max_q) fail(E8QC_EINVAL, "batch larger than the plan's max_queries");
    const e8qc_plan::Graph* g = nullptr;
    for (const auto& gg : P->graphs)
        if (gg.nq >= nq) {
            g = &gg;
            break;
        }
    if (!g) fail(E8QC_ESTATE, "plan has no captured size for this batch");
    E8QC_CUDA(cudaEventSynchronize(P->staged));  // the previous run has read the staging
    for (size_t i = 0; i < nq; ++i) {
        if (k[i] == 0 || k[i] > P->k_max) fail(E8QC_EINVAL, "k must be in [1, k_max]");
        if (nprobe[i] == 0 || nprobe[i] > P->np_max) fail(E8QC_EINVAL, "nprobe must be in [1, nprobe_max]");
        P->hk[i] = k[i];
        P->hnp[i] = static_cast<uint32_t>(std::min<size_t>(nprobe[i], P->nlist));
    }
    for (size_t i = nq; i < g->nq; ++i) P->hk[i] = P->hnp[i] = 1u;
    E8QC_CUDA(cudaMemcpyAsync(P->q.p, queries, nq * P->dim * 4, cudaMemcpyDefault, s));
    if (g->nq > nq) E8QC_CUDA(cudaMemsetAsync(P->q.as<float>() + nq * P->dim, 0, (g->nq - nq) * P->dim * 4, s));
    E8QC_CUDA(cudaMemcpyAsync(P->k.p, P->hk, g->nq * 4, cudaMemcpyHostToDevice, s));
    E8QC_CUDA(cudaMemcpyAsync(P->np.p, P->hnp, g->nq * 4, cudaMemcpyHostToDevice, s));
    E8QC_CUDA(cudaEventRecord(P->staged, s));
    E8QC_CUDA(cudaGraphLaunch(g->exec, s));
    E8QC_CUDA(cudaMemcpyAsync(out_ids, P->ids.p, nq * P->k_max * 4, cudaMemcpyDefault, s));
    if (out_dists) E8QC_CUDA(cudaMemcpyAsync(out_dists, P->d.p, nq * P->k_max * 4, cudaMemcpyDefault, s));
}

// Synchronise s and report a kernel wait timeout of the plan's last runs.
void plan_check(e8qc_plan* P, cudaStream_t s) { P->ws.check_error(s); }

size_t plan_max_queries(const e8qc_plan* P) { return P->max_q; }

uint64_t plan_kernels(const e8qc_plan* P) { return P->kernels; }

void plan_free(e8qc_plan* P) {
    if (!P) return;
    int prev = 0;
    const bool have_prev = cudaGetDevice(&prev) == cudaSuccess;
    cudaSetDevice(P->device);
    cudaStreamSynchronize(P->cs);
    cudaEventSynchronize(P->staged);
    delete P;
    if (have_prev) cudaSetDevice(prev);
}

// Create a plan (see e8qc_plan_create); throws on failure.
e8qc_plan* plan_make(std::shared_ptr<SearchTarget> t, int mode, size_t max_q, size_t k_max, size_t np_max,
                     bool autotune, bool exact_size) {
    t->check_mode(mode);
    if (max_q == 0) fail(E8QC_EINVAL, "max_queries must be positive");
    if (k_max == 0 || k_max > static_cast<size_t>(kMaxK)) fail(E8QC_EINVAL, "k_max must be in [1, 128]");
    if (np_max == 0) fail(E8QC_EINVAL, "nprobe_max must be positive");
    auto P = std::make_unique<e8qc_plan>();
    P->target = t;
    P->mode = mode;
    P->dim = t->dim;
    P->nlist = t->nlist;
    P->device = t->device;
    P->max_q = max_q;
    P->k_max = k_max;
    P->np_max = std::min(np_max, P->nlist);
    int prev = 0;
    E8QC_CUDA(cudaGetDevice(&prev));
    E8QC_CUDA(cudaSetDevice(P->device));
    struct Restore {
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{prev};
    t->prepare(mode);
    P->ws.device = P->device;
    E8QC_CUDA(cudaStreamCreateWithFlags(&P->cs, cudaStreamNonBlocking));
    E8QC_CUDA(cudaEventCreateWithFlags(&P->staged, cudaEventDisableTiming));
    E8QC_CUDA(cudaEventRecord(P->staged, P->cs));
    E8QC_CUDA(cudaMallocHost(reinterpret_cast<void**>(&P->hk), max_q * 4));
    E8QC_CUDA(cudaMallocHost(reinterpret_cast<void**>(&P->hnp), max_q * 4));
    P->q.alloc(max_q * P->dim * 4);
    P->k.alloc(max_q * 4);
    P->np.alloc(max_q * 4);
    P->ids.alloc(max_q * k_max * 4);
    P->d.alloc(max_q * k_max * 4);
    std::vector<size_t> sizes;
    if (!exact_size)
        for (size_t n = 64; n < max_q; n <<= 1) sizes.push_back(n);
    sizes.push_back(max_q);
    std::sort(sizes.rbegin(), sizes.rend());
    cudaStream_t s = P->cs;
    for (size_t n : sizes) {
        int sched = 0, stages = 6;
        if (autotune) {
            t->autotune(P->ws, mode, n, k_max, P->np_max, s, &sched, &stages);
        } else {
            t->stored_tuning(P->ws, mode, n, P->np_max);
            sched = P->ws.sched;
            stages = P->ws.stages;
        }
        P->ws.sched = sched;
        P->ws.stages = stages;
        // worst-case shape of this size: every row at k_max / nprobe_max
        for (size_t i = 0; i < n; ++i) {
            P->hk[i] = static_cast<uint32_t>(k_max);
            P->hnp[i] = static_cast<uint32_t>(P->np_max);
        }
        E8QC_CUDA(cudaMemsetAsync(P->q.p, 0, n * P->dim * 4, s));
        E8QC_CUDA(cudaMemcpyAsync(P->k.p, P->hk, n * 4, cudaMemcpyHostToDevice, s));
        E8QC_CUDA(cudaMemcpyAsync(P->np.p, P->hnp, n * 4, cudaMemcpyHostToDevice, s));
        auto enqueue = [&] {
            const uint64_t kn = t->enqueue(P->ws, mode, P->q.as<float>(), n, P->k.as<uint32_t>(),
                                           P->np.as<uint32_t>(), k_max, P->np_max, P->ids.as<uint32_t>(),
                                           P->d.as<float>(), s, false);
            if (n == max_q) P->kernels = kn;
        };
        enqueue();  // sizes the workspace, sets kernel attributes
        P->ws.check_error(s);
        cudaGraph_t graph = nullptr;
        E8QC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue();
        } catch (...) {
            cudaStreamEndCapture(s, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        E8QC_CUDA(cudaStreamEndCapture(s, &graph));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        E8QC_CUDA(ie);
        P->graphs.push_back(e8qc_plan::Graph{n, exec, sched, stages});
    }
    std::sort(P->graphs.begin(), P->graphs.end(),
              [](const e8qc_plan::Graph& a, const e8qc_plan::Graph& b) { return a.nq < b.nq; });
    E8QC_CUDA(cudaStreamSynchronize(s));
    return P.release();
}

}  // namespace e8qc

namespace {
int guard(const std::function<void()>& f) {
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

extern "C" int e8qc_plan_create(e8qc_index* idx, int mode, size_t max_queries, size_t k_max, size_t nprobe_max,
                                int autotune, e8qc_plan** out) {
    return guard([&] {
        if (!idx || !out) fail(E8QC_EINVAL, "null argument");
        *out = plan_make(e8q_target(idx), mode, max_queries, k_max, nprobe_max, autotune != 0);
    });
}

extern "C" int e8qc_plan_create_me8q(e8qc_me8q* idx, int mode, size_t max_queries, size_t k_max, size_t nprobe_max,
                                     int autotune, e8qc_plan** out) {
    return guard([&] {
        if (!idx || !out) fail(E8QC_EINVAL, "null argument");
        *out = plan_make(me8q_target(idx), mode, max_queries, k_max, nprobe_max, autotune != 0);
    });
}

extern "C" int e8qc_plan_run(e8qc_plan* P, const float* queries, size_t nq, const uint32_t* k, const uint32_t* nprobe,
                             uint32_t* out_ids, float* out_dists, void* stream) {
    return guard([&] {
        if (!P) fail(E8QC_EINVAL, "null plan");
        if (nq == 0) return;
        if (!queries || !k || !nprobe || !out_ids) fail(E8QC_EINVAL, "null buffer");
        if (is_device_ptr(k) || is_device_ptr(nprobe)) fail(E8QC_EINVAL, "k and nprobe must be host arrays");
        int prev = 0;
        E8QC_CUDA(cudaGetDevice(&prev));
        E8QC_CUDA(cudaSetDevice(P->device));
        struct Restore {
            int d;
            ~Restore() { cudaSetDevice(d); }
        } restore{prev};
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        plan_enqueue(P, queries, nq, k, nprobe, out_ids, out_dists, s);
        plan_check(P, s);
    });
}

extern "C" int e8qc_plan_destroy(e8qc_plan* P) {
    return guard([&] {
        if (!P) return;
        cudaSetDevice(P->device);
        cudaStreamSynchronize(P->cs);
        cudaEventSynchronize(P->staged);
        delete P;
    });
}
