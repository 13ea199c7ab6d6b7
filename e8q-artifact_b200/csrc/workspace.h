// Device buffers and the per-index search workspace.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>

#include "internal.h"

namespace e8qc {

// Owning device allocation (cudaMalloc / cudaFree), grown on demand.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void alloc(size_t b) {
        release();
        if (b == 0) b = 16;
        E8QC_CUDA(cudaMalloc(&p, b));
        bytes = b;
    }
    void ensure(size_t b) {
        if (b > bytes) alloc(b);
    }
    void upload(const void* src, size_t b, cudaStream_t s) {
        alloc(b);
        if (b) E8QC_CUDA(cudaMemcpyAsync(p, src, b, cudaMemcpyHostToDevice, s));
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

// Scratch the search paths reuse across calls (one per index; calls on an
// index are serialised). Counters used by last-CTA-done merges are zeroed at
// allocation and reset by the kernels themselves.
struct Workspace {
    int device = 0;
    DevBuf rq;  // nq*pd rotated queries
    // staging of host-buffer calls: queries, per-query k / nprobe, results
    DevBuf stage_q, stage_k, stage_np, stage_ids, stage_d;
    size_t rq_cap = 0;
    // plain path
    DevBuf keys, probes, probe_d2, tile_off, probe_info, route_counter, total_tiles;
    size_t route_cap = 0;
    DevBuf part_d, part_id, scan_counter;
    size_t scan_cap = 0;
    DevBuf err;  // device error word written by bounded waits
    uint32_t* err_host = nullptr;
    // batched path (grown on demand by batched_search)
    DevBuf b_keys, b_qn2, b_probes, b_pd2, b_pos, b_pair_q, b_pair_d2, b_cnt, b_off, b_fill, b_items,
        b_nitems, b_part_d, b_part_id;
    // precision path: int8 queries, per-query scale and sum, per-list row
    // bases, the proxy-distance rows and the gathered int8 query rows
    DevBuf p_q8, p_scale, p_sum, p_rowbase, p_prox, p_a8, p_pscale, p_cand;
    // tensor-core routing: int8 slice planes and per-row scale / norms of the
    // queries and the centroids
    DevBuf r_qplane, r_cplane, r_qmeta, r_cmeta, r_ub;
    // pruned path: candidate/survivor counts, per-query final k-th distances,
    // and per group of queries the tile offsets and the probed rows' coarse
    // values (LUT sum, bound terms)
    DevBuf pr_stats, pr_thr, p2_toff, p2_acc, p2_P, p2_perp;
    size_t pr_thr_cap = 0, pr_last_nq = 0;
    // pruned paths' per-query u8 LUTs and scalars (both indexes), and the
    // ME8Q path's LUT steps, thresholds and candidate / survivor counts
    DevBuf f_lut, f_qrun, f_delta, f_thr, f_counts;
    // tuning of the grouped paths (chosen by the autotuner): work-queue order
    // (0: longest list first, 1: list id order) and the precision scan's
    // shared-memory ring depth (4, 6 or 8 K-chunk stages)
    int sched = 0;
    int stages = 6;
    // batch routing on the int8 tensor cores (route_tc) where it applies
    bool route_tc = true;
    // optional CUDA events around the batched / precision scan kernel (set by
    // the caller while profiling; recorded on the launch stream)
    cudaEvent_t scan_ev0 = nullptr, scan_ev1 = nullptr;
    void mark_scan(bool end, cudaStream_t s) {
        cudaEvent_t e = end ? scan_ev1 : scan_ev0;
        if (e) E8QC_CUDA(cudaEventRecord(e, s));
    }
    // the same around the precision path's select + rescore kernel
    cudaEvent_t final_ev0 = nullptr, final_ev1 = nullptr;
    // and around the routing + grouping stage (route GEMM, select, items, scatter)
    cudaEvent_t prep_ev0 = nullptr, prep_ev1 = nullptr;
    void mark_prep(bool end, cudaStream_t s) {
        cudaEvent_t e = end ? prep_ev1 : prep_ev0;
        if (e) E8QC_CUDA(cudaEventRecord(e, s));
    }
    void mark_final(bool end, cudaStream_t s) {
        cudaEvent_t e = end ? final_ev1 : final_ev0;
        if (e) E8QC_CUDA(cudaEventRecord(e, s));
    }

    ~Workspace() {
        if (err_host) cudaFreeHost(err_host);
    }
    void ensure_err() {
        if (err.p) return;
        err.alloc(4);
        E8QC_CUDA(cudaMemset(err.p, 0, 4));
        E8QC_CUDA(cudaMallocHost(&err_host, 4));
    }
    // Synchronise the stream and turn a kernel-reported wait timeout into an
    // error (the word is cleared for the next call).
    void check_error(cudaStream_t s) {
        ensure_err();
        E8QC_CUDA(cudaMemcpyAsync(err_host, err.p, 4, cudaMemcpyDeviceToHost, s));
        E8QC_CUDA(cudaStreamSynchronize(s));
        if (*err_host != 0) {
            E8QC_CUDA(cudaMemsetAsync(err.p, 0, 4, s));
            E8QC_CUDA(cudaStreamSynchronize(s));
            fail(E8QC_ETIMEOUT, "a bounded device wait gave up (a bulk copy or barrier did not complete in time)");
        }
    }
    void ensure_queries(size_t nq, size_t pd) {
        if (nq * pd > rq_cap) {
            rq.alloc(nq * pd * sizeof(float));
            rq_cap = nq * pd;
        }
    }
    void ensure_route(size_t nlist) {
        if (nlist <= route_cap) return;
        keys.alloc(nlist * 8);
        probes.alloc(nlist * 4);
        probe_d2.alloc(nlist * 4);
        tile_off.alloc((nlist + 1) * 4);
        probe_info.alloc(nlist * 8);
        route_counter.alloc(4);
        total_tiles.alloc(4);
        E8QC_CUDA(cudaMemset(route_counter.p, 0, 4));
        route_cap = nlist;
    }
    void ensure_pruned(size_t nq) {
        ensure_err();
        if (!pr_stats.p) pr_stats.alloc(16);
        if (nq > pr_thr_cap) {
            pr_thr.alloc(nq * 4);
            pr_thr_cap = nq;
        }
    }
    void ensure_scan(size_t grid) {
        ensure_err();
        if (grid <= scan_cap) return;
        part_d.alloc(grid * kMaxK * 4);
        part_id.alloc(grid * kMaxK * 4);
        scan_counter.alloc(4);
        E8QC_CUDA(cudaMemset(scan_counter.p, 0, 4));
        scan_cap = grid;
    }
};

// Batched search over nq rotated queries (batched.cu). k_arr / np_arr are
// optional per-query device arrays (NULL = uniform k / nprobe). Output rows
// are out_stride wide. Returns the number of kernels launched.
int batched_search(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq,
                   const uint32_t* k_arr, const uint32_t* np_arr, size_t k, size_t nprobe,
                   size_t out_stride, uint32_t* out_ids, float* out_d, size_t max_tiles,
                   cudaStream_t s);

// Route + per-query select + grouping of (query, list) pairs into work items
// of up to qt queries per list (shared by the batched and precision paths).
// Each list's pairs start at a multiple of `align` (unused slots hold query
// id UINT32_MAX); partial-result buffers hold part_width entries per pair.
// Returns the number of kernels launched.
int batched_prepare(const DevIndex& ix, Workspace& ws, const float* rq, size_t nq, const uint32_t* np_arr,
                    size_t nprobe, size_t part_width, int qt, int align, cudaStream_t s);

}  // namespace e8qc
