// Plain search that allocates nothing: e8qc_e8q_search_plain_noalloc.
//
// Some callers cannot let this library allocate device memory during a
// search: a serving process whose HBM is already reserved by its framework's
// caching allocator (an extra cudaMalloc fails or fragments that pool), a
// request handler that must not stall other streams (cudaFree synchronises
// the whole device), or a foreign-language host (JNI, cgo) that owns a fixed
// memory budget. This entry point runs the same kernels as the plain search
// (rotation, routing, streaming scan with its top-k merge) but takes its
// scratch from the file-scope array below instead of the index's workspace,
// and the caller passes device buffers for the queries and the results, so
// nothing is staged either.
//
// The array is a fixed 3.0 MB per device that loads the library and stays
// allocated until the process exits. Its size sets the limits checked on every
// call: at most kNaMaxLists lists and kNaMaxPd padded dimensions. The first
// call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture. Every call reuses the same array and it keeps
// the last call's contents: the counters the kernels rely on are cleared at
// the start of each call, and calls whose GPU work overlaps (two host
// threads with different indexes, or two streams) race on the array and must
// be serialised by the caller. A call holds its index's mutex until its
// kernels have finished (it waits for its stream before returning), so a
// build or load of the same index cannot replace the buffers it reads.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "e8qc.h"
#include "internal.h"
#include "scan_plain.h"

namespace e8qc {

// Index internals the entry point needs (index.cpp).
std::unique_lock<std::mutex> plain_context(e8qc_index* x, size_t nprobe, DevIndex* view, int* device,
                                           size_t* nlist, size_t* dim, size_t* max_tiles);
bool is_device_ptr_on(const void* p, int device);
void set_last_error(const std::string& s);

namespace {

constexpr size_t kNaMaxLists = 65536;
constexpr size_t kNaMaxPd = 4096;
constexpr int kNaMaxGrid = 1024;

struct NaScratch {
    uint64_t keys[kNaMaxLists];
    uint32_t probes[kNaMaxLists];
    float probe_d2[kNaMaxLists];
    uint32_t tile_off[kNaMaxLists + 1];
    uint2 probe_info[kNaMaxLists];
    float rq[kNaMaxPd];
    float part_d[kNaMaxGrid * kMaxK];
    uint32_t part_id[kNaMaxGrid * kMaxK];
    uint32_t words[4];  // route counter, scan counter, total tiles, error word
};

static __device__ __align__(256) NaScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch per device ordinal (host code may not
// use the symbol itself as an address).
NaScratch* scratch_for(int device) {
    static std::mutex mu;
    static NaScratch* ptrs[64] = {};
    if (device < 0 || device >= 64) fail(E8QC_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (ptrs[device] == nullptr) {
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (rc != cudaSuccess || p == nullptr)
            fail(E8QC_ECUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(rc));
        ptrs[device] = static_cast<NaScratch*>(p);
    }
    return ptrs[device];
}

}  // namespace
}  // namespace e8qc

using namespace e8qc;

extern "C" int e8qc_e8q_search_plain_noalloc(e8qc_index* idx, const float* queries, size_t nq, size_t k,
                                             size_t nprobe, uint32_t* out_ids, float* out_dists, void* stream) {
    try {
        if (k == 0) fail(E8QC_EINVAL, "k must be positive");
        if (k > static_cast<size_t>(kMaxK)) fail(E8QC_EINVAL, "k must be <= 128");
        if (nprobe == 0) fail(E8QC_EINVAL, "nprobe must be positive");
        DevIndex view{};
        int device = 0;
        size_t nlist = 0, dim = 0, max_tiles = 0;
        // held until the kernels below have finished
        const std::unique_lock<std::mutex> index_lock =
            plain_context(idx, nprobe, &view, &device, &nlist, &dim, &max_tiles);
        if (nq == 0) return E8QC_OK;
        if (nlist > kNaMaxLists)
            fail(E8QC_EINVAL, "no-alloc search supports at most 65536 lists (the scratch array's size)");
        if (static_cast<size_t>(view.pd) > kNaMaxPd)
            fail(E8QC_EINVAL, "no-alloc search supports padded_dim <= 4096 (the scratch array's size)");
        int prev = 0;
        E8QC_CUDA(cudaGetDevice(&prev));
        if (prev != device) E8QC_CUDA(cudaSetDevice(device));
        struct Restore {
            int d;
            ~Restore() { cudaSetDevice(d); }
        } restore{prev};
        if (!is_device_ptr_on(queries, device) || !is_device_ptr_on(out_ids, device) ||
            !is_device_ptr_on(out_dists, device))
            fail(E8QC_EINVAL, "no-alloc search needs device pointers for queries, ids and dists, on the index's device");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        NaScratch* sc = scratch_for(device);
        const size_t np = nprobe < nlist ? nprobe : nlist;
        int sms = 148;
        E8QC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        // one CTA per SM but one (the routing kernel's last CTA keeps its SM)
        const size_t cap = static_cast<size_t>(sms > 1 ? sms - 1 : 1);
        int grid = static_cast<int>(max_tiles < cap ? max_tiles : cap);
        if (grid < 1) grid = 1;
        if (grid > kNaMaxGrid) grid = kNaMaxGrid;
        // counters and the error word must start at zero on every call
        E8QC_CUDA(cudaMemsetAsync(sc->words, 0, sizeof(sc->words), s));
        RouteWork rw{sc->keys, sc->probes, sc->probe_d2, sc->tile_off, &sc->words[0], &sc->words[2], sc->probe_info};
        ScanWork sw{sc->part_d, sc->part_id, &sc->words[1], &sc->words[3], grid};
        const ScanGeo geo = plain_scan_geo(view, (max_tiles + static_cast<size_t>(grid) - 1) / static_cast<size_t>(grid));
        for (size_t i = 0; i < nq; ++i) {
            launch_rotate(view, queries + i * dim, 1, sc->rq, s);
            launch_route_one(view, sc->rq, static_cast<int>(np), rw, s);
            launch_scan_plain(view, sc->rq, rw, static_cast<int>(np), static_cast<int>(k), sw, geo, out_ids + i * k,
                              out_dists + i * k, s);
        }
        // results are complete when the call returns (and the index mutex
        // may be released): wait for the stream
        E8QC_CUDA(cudaStreamSynchronize(s));
        return E8QC_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return E8QC_EINVAL;
    }
}
