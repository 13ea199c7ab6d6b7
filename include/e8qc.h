/* e8qc.h -- C ABI of the B200 (sm_100a) E8Q IVF search library (libe8qcuda.so).
 *
 * Plain C types only: pointers, sizes, status codes. No exception crosses this
 * boundary; every function returns E8QC_OK (0) or a negative E8QC_E* code and
 * leaves a message in e8qc_last_error() (thread-local).
 *
 * Memory: the index owns all of its device memory. Buffers passed in are the
 * caller's and may be HOST or DEVICE pointers (device pointers must belong to
 * the index's device; the library tells them apart with
 * cudaPointerGetAttributes). Host buffers are copied in/out inside the call.
 * `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 * stream); calls return after the results are in the caller's buffers.
 *
 * Threading: an index may be shared by host threads; calls on one index are
 * serialised internally (the index owns one search workspace).
 *
 * Reference interfaces replaced (paths in the reference project):
 *   python_bindings/e8q_bindings.cpp:22-344   E8qIndex pybind11 class
 *   include/e8qlib/index/e8q.hpp:121-187      E8qIndex C++ class
 *   include/e8qlib/quantization/e8q_codec.hpp:48-146  codec helpers
 */
#ifndef E8QC_H
#define E8QC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define E8QC_OK 0
#define E8QC_EINVAL -1   /* bad argument: std::invalid_argument -> ValueError */
#define E8QC_ESTATE -2   /* wrong state (not built, ...): std::runtime_error */
#define E8QC_ECUDA -3    /* CUDA runtime error */
#define E8QC_ENOMEM -4   /* device or host allocation failed */
#define E8QC_ERANGE -5   /* unknown id: std::out_of_range / invalid_argument */
#define E8QC_EIO -6      /* file I/O or format error */
#define E8QC_ETIMEOUT -7 /* a bounded device wait gave up, or a served request expired */
#define E8QC_ECANCELED -8 /* a served request was canceled (e8qc_server_cancel) */

/* Search modes. PLAIN is the drop-in: one query per launch sequence
 * (rotate -> route -> streaming scan -> top-k), every candidate of every probed
 * list scored exactly. BATCHED groups a whole query batch by probed list and
 * runs the persistent work-queue kernel (same estimator, same results within
 * fp32 rounding). */
#define E8QC_MODE_PLAIN 0
#define E8QC_MODE_BATCHED 1
/* PRECISION (an addition of this library, no counterpart in the reference):
 * batch grouped by list as in BATCHED, but candidates are generated on the
 * INT8 tensor cores from an int8 plane of every vector's levels (built on the
 * first precision search, padded_dim bytes per vector) and int8 queries; each
 * query's best max(32, 3k) (at most 128) proxy candidates are then rescored
 * with the exact estimator. Distances returned are exact; recall against the
 * exact scan is measured, not guaranteed. */
#define E8QC_MODE_PRECISION 2
/* PRUNED is the reference's production search (E8qIndex::Search with its
 * coarse gate, src/index/e8q_search.cpp:215-293): a coarse pass prices one
 * rowA byte per 8-dim block against the query's u8 LUT (PrepareQuery), the
 * zero-parallel-residual bound of the scan banks rejects vectors (and whole
 * 32-row batches) that cannot beat the running heap's k-th distance, and the
 * survivors are staged 32 at a time and scored exactly. One warp per query
 * takes these decisions in the reference's order against the same heap, so
 * the survivors and results are the reference's; the bound, its LUT and
 * banks and prune_alpha are the reference's. Throughput comes from the batch
 * (one query alone is one warp's work). With set_disable_prune every
 * candidate is scored (the reference's plain scan). stats: candidates scanned
 * and survivors refined. On an ME8Q index (e8qc_me8q_search_mode) the mode
 * replays the reference's FastScan cascade the same way. */
#define E8QC_MODE_PRUNED 3

/* Maximum top-k (include/e8qlib/index/e8q.hpp:44 kMaxK). */
#define E8QC_MAX_K 128

typedef struct e8qc_index e8qc_index;

/* Per-call counters; mirrors e8qlib::SearchStats (include/e8qlib/index/e8q.hpp:55-62)
 * plus device timings (CUDA events, microseconds summed over the call). */
typedef struct e8qc_stats {
    uint64_t candidates; /* vectors scored */
    uint64_t survivors;  /* vectors that reached the exact estimator (all, in plain mode) */
    double rotate_us;
    double route_us;
    double scan_us;
    double refine_us;
    uint64_t launches;   /* kernels this library launched for the call */
} e8qc_stats;
/* A grouped-mode search of 1,024 or more host-resident queries whose mode,
   size, k and nprobe repeat the previous call's replays a captured graph of
   that shape
   (the index then holds a second workspace for it, released when the shape
   changes or the index is rebuilt); its stats carry the graph's kernel count
   and its whole device time, staging copies included, as scan_us. */

/* The final pruning threshold of each query of the last E8QC_MODE_PRUNED
 * search on this index (its first nq queries): the running heap's k-th
 * distance at the end, +inf where fewer than k candidates survived. No
 * reference counterpart; for checking the bound. */
int e8qc_e8q_pruned_thresholds(e8qc_index* idx, float* out, size_t nq);

typedef struct e8qc_info {
    uint64_t dim, padded_dim, n, nlist, memory_bytes;
    int32_t nbits, device, built, disable_prune;
    float prune_alpha;
} e8qc_info;

/* ---- errors / library ---------------------------------------------------- */
const char* e8qc_last_error(void);
int e8qc_version(void);

/* ---- codec (include/e8qlib/quantization/e8q_codec.hpp) -------------------- */
/* BranchLevels(bits, branch) (e8q_codec.hpp:50-52): 2^bits doubles. */
int e8qc_branch_levels(int bits, int branch, double* out);
/* FixedScale(bits) (e8q_codec.hpp:48). */
int e8qc_fixed_scale(int bits, double* out);
/* EncodeVectorAtScale(unit, padded_dim, bits, FixedScale(bits)) for n vectors
 * on the GPU (e8q_codec.hpp:90-100). unit: n*padded_dim floats; digits:
 * n*(padded_dim/8)*8 uint16; branch: n*(padded_dim/8) uint8. Bit-exact. */
int e8qc_encode(int device, int bits, const float* unit, size_t n, size_t padded_dim,
                uint16_t* digits, uint8_t* branch, void* stream);
/* FhtKac4Rotator(dim, seed).Rotate for n rows (include/e8qlib/utils/rotator.hpp:17-42)
 * on the GPU: src n*dim floats -> dst n*padded_dim floats. Bit-exact. */
int e8qc_rotate(int device, size_t dim, uint64_t seed, const float* src, size_t n, float* dst,
                void* stream);

/* ---- E8Q index (python_bindings/e8q_bindings.cpp, index/e8q.hpp) ---------- */
/* E8qIndex(dim, nbits, seed) (e8q_bindings.cpp:24-32): nbits in [1, 13]. */
int e8qc_e8q_create(int device, size_t dim, int nbits, uint64_t seed, e8qc_index** out);
int e8qc_e8q_destroy(e8qc_index* idx);
/* E8qIndex::Build (e8q.hpp:123-134; e8q_bindings.cpp:34-72). data n*dim,
 * centroids nlist*dim, cluster_ids n (each < nlist). Encoding runs on the GPU
 * with codes bit-exact to the reference encoder. */
int e8qc_e8q_build(e8qc_index* idx, const float* data, size_t n, const float* centroids,
                   size_t nlist, const uint32_t* cluster_ids, float prune_alpha, void* stream);
/* E8qIndex::Search for nq queries (e8q.hpp:139-143; e8q_bindings.cpp:74-169):
 * out_ids / out_dists nq*k, ascending (distance, id); unused slots are
 * UINT32_MAX / +inf. 0 < k <= E8QC_MAX_K, nprobe > 0 (clamped to nlist). */
int e8qc_e8q_search(e8qc_index* idx, const float* queries, size_t nq, size_t k, size_t nprobe,
                    int mode, uint32_t* out_ids, float* out_dists, e8qc_stats* stats,
                    void* stream);
/* Serving form: per-query k[i] and nprobe[i]; output row i holds k[i] results
 * padded to k_max with UINT32_MAX / +inf. Uses the batched kernel. */
int e8qc_e8q_search_ragged(e8qc_index* idx, const float* queries, size_t nq,
                           const uint32_t* k, const uint32_t* nprobe, size_t k_max,
                           uint32_t* out_ids, float* out_dists, e8qc_stats* stats,
                           void* stream);
/* Ragged search with an explicit mode (E8QC_MODE_BATCHED or
 * E8QC_MODE_PRECISION); e8qc_e8q_search_ragged is this with BATCHED. An
 * addition of this library: the serving loop's entry for mixed batches. */
int e8qc_e8q_search_ragged_mode(e8qc_index* idx, const float* queries, size_t nq, const uint32_t* k,
                                const uint32_t* nprobe, size_t k_max, int mode, uint32_t* out_ids,
                                float* out_dists, e8qc_stats* stats, void* stream);
/* E8qIndex::Estimate (e8q.hpp:151-152): estimated squared L2 of stored id. */
int e8qc_e8q_estimate(e8qc_index* idx, const float* query, uint32_t id, float* out);
/* E8qIndex::SetDisablePrune / SetPruneAlpha (e8q.hpp:173-180). The GPU paths
 * score every candidate exactly; the flags are kept and reported. */
int e8qc_e8q_set_disable_prune(e8qc_index* idx, int on);
int e8qc_e8q_set_prune_alpha(e8qc_index* idx, float alpha);
int e8qc_e8q_info(const e8qc_index* idx, e8qc_info* out);
/* Scan-kernel profile: while enabled, every call records CUDA events around
 * each launch of the dominant scan kernel on the call's stream and counts the
 * candidates it scored (plain mode reads the probe lists back once per query,
 * so timings of the calls themselves are perturbed). enable=1 resets and
 * starts; enable=0 stops and fills *out (may be NULL). */
typedef struct e8qc_profile {
    uint64_t scan_launches;  /* dominant-kernel launches timed */
    double scan_ms;          /* summed CUDA-event time of those launches */
    uint64_t candidates;     /* (query, vector) pairs scored */
    uint64_t algo_bytes;     /* plain: candidates * (bits*padded_dim/8 + 8), codes + g1/h3; batched:
                                list_once * (bits*padded_dim/8 + 8); precision: list_once *
                                (padded_dim + 8) int8 proxies + g1/h3, plus 2 per candidate written */
    uint64_t queries;
    uint64_t list_vectors;   /* vectors read by the work items (batched modes: once per work item) */
    uint64_t list_once;      /* vectors of the probed lists, each list counted once per call */
    uint64_t item_bytes;     /* algo_bytes with list_vectors in place of list_once (what the work
                                items request; repeats of a list are mostly served by L2) */
    uint64_t final_launches; /* precision mode: select + rescore kernel launches timed */
    double final_ms;         /* their summed CUDA-event time */
    uint64_t final_bytes;    /* their algorithmic bytes: 2 per proxy distance read + per query
                                C * (bits*padded_dim/8 + 12) for the rescored candidates */
    double prep_ms;          /* precision mode: routing + grouping (route GEMM, probe select,
                                work items, pair scatter); plain mode: the per-query routing
                                launches; summed CUDA-event time */
} e8qc_profile;
int e8qc_e8q_profile(e8qc_index* idx, int enable, e8qc_profile* out);
/* Plain search that allocates nothing (no counterpart in the reference; an
 * addition of this library). For callers that cannot let a search allocate
 * device memory: a serving process whose HBM is reserved by its framework's
 * caching allocator, a request handler that must not stall other streams
 * (cudaFree synchronises the device), a JNI/cgo host with a fixed memory
 * budget. Same kernels and results as e8qc_e8q_search(..., E8QC_MODE_PLAIN),
 * but the scratch is a fixed 3.0 MB static device array per device (held
 * until the process exits) and queries (nq*dim), out_ids and out_dists
 * (nq*k) must be DEVICE pointers on the index's device (else E8QC_EINVAL).
 * Limits: nlist <= 65536, padded_dim <= 4096; larger indexes return
 * E8QC_EINVAL. The first call on a device resolves the array's address (make
 * it before any stream capture). All calls share the array: calls whose GPU
 * work overlaps race and must be serialised by the caller. The call holds the
 * index's mutex and waits for `stream` before returning, so the results are
 * in out_ids / out_dists when it returns. */
int e8qc_e8q_search_plain_noalloc(e8qc_index* idx, const float* queries, size_t nq, size_t k,
                                  size_t nprobe, uint32_t* out_ids, float* out_dists, void* stream);
/* INT8 tensor-core self-test / throughput probe (no reference counterpart):
 * C[128 x n] = A[128 x k] * B[n x k]^T (int8 x int8 -> int32, K-major rows)
 * through tcgen05 kind::i8 with the accumulator in TMEM; `grid` CTAs each
 * repeat the product `reps` times (CTA 0 writes C); *ms = kernel time.
 * n: multiple of 16 in [16, 256]; k: multiple of 32 in [32, 256]. */
int e8qc_tc_i8_gemm(int device, const int8_t* A, const int8_t* B, int n, int k, int reps, int grid,
                    int32_t* C, float* ms);
/* E8qIndex::Load (src/index/e8q_io.cpp:86-211): open an index file the
 * reference wrote with E8qIndex::Save (E8AX layout, optional build-options
 * trailer) straight into a device index on `device`. Codes, g1/h3, ids,
 * rotator, rotated mean and centroids come from the file (nothing is
 * re-encoded); the file's pruning headers are not needed by the device scans.
 * E8QC_EIO for an unreadable, foreign, truncated or inconsistent file. */
int e8qc_e8q_load(int device, const char* path, e8qc_index** out);
/* Save as an E8AX file the reference's E8qIndex::Load reads (E8qIndex::Save,
   src/index/e8q_io.cpp:35-84): a built index writes the scan banks from its
   build, a loaded one the banks it read. */
int e8qc_e8q_save(const e8qc_index* idx, const char* path);
/* Copy the global ids, cluster-major (n entries), to a host buffer. */
int e8qc_e8q_get_ids(const e8qc_index* idx, uint32_t* out);
/* Export the per-vector lattice codes (cluster-major, the order of
 * e8qc_e8q_get_ids) to host buffers: digits n*B*8 uint16, branch n*B uint8,
 * g1 n, h3 n (any may be NULL). B = padded_dim/8. */
int e8qc_e8q_export_codes(const e8qc_index* idx, uint16_t* digits, uint8_t* branch, float* g1,
                          float* h3);

/* ---- ME8Q: mixed-rate index (e8qlib::me8q::Me8qIndex, include/e8qlib/index/me8q.hpp:66-140) ---- */
typedef struct e8qc_me8q e8qc_me8q;
/* BuildOptions (me8q.hpp:31-52) plus the optional per-dimension variance of
 * Build (me8q.hpp:76-80). plan_spec "L:B,L:B,..." (runs of 64-dim multiples
 * covering the padded dim) overrides the DP plan; max_bits <= 0 means 13.
 * prune_alpha is accepted for interface parity: the device scan scores every
 * vector of the probed lists exactly, so results do not depend on it. */
typedef struct e8qc_me8q_build_opts {
    const float* variance; /* dim floats, host or device; NULL: computed from data */
    const char* plan_spec; /* NULL or "": DP plan */
    int drop_energy;       /* add the dropped dims' residual energy to the last run's h2 */
    float prune_alpha;
    double extra_budget_bits;
    int max_bits;
} e8qc_me8q_build_opts;
typedef struct e8qc_me8q_meta {
    uint64_t n, dim, padded_dim, nlist, nruns, ncoded, route_dim, bytes_per_vector, memory_bytes;
    double bits_per_dim; /* 8 * bytes_per_vector / dim (me8q_io.cpp:176-181) */
    float avg_bits;
    int is_built;
} e8qc_me8q_meta;
/* Allocate (src/quantization/me8q_plan.cpp:47-167): SAQ's DP plan for a
 * per-dimension variance padded to padded_dim (a multiple of 64). Host only.
 * *count runs; up to cap (len, bits) pairs written. */
int e8qc_me8q_allocate(const float* var_padded, size_t padded_dim, float avg_bits, int max_bits,
                       double extra_budget_bits, size_t* lens, int* bits, size_t cap, size_t* count);
/* detail::ParsePlanSpec (src/index/me8q_common.cpp:37-68): "L:B,..." with
 * L a positive multiple of 64, B in [0, 13], lens summing to padded_dim;
 * E8QC_EINVAL otherwise. Host only. */
int e8qc_me8q_parse_plan(const char* spec, size_t padded_dim, size_t* lens, int* bits, size_t cap, size_t* count);
/* Me8qIndex(dim, avg_bits, seed): seed 0 keeps the default rotator seed. */
int e8qc_me8q_create(int device, size_t dim, float avg_bits, uint64_t seed, e8qc_me8q** out);
int e8qc_me8q_destroy(e8qc_me8q* idx);
/* Me8qIndex::Build (me8q_build.cpp:42-311): data n x dim, centroids nlist x
 * dim, cluster_ids n; host or device pointers; opts may be NULL. */
int e8qc_me8q_build(e8qc_me8q* idx, const float* data, size_t n, const float* centroids, size_t nlist,
                    const uint32_t* cluster_ids, const e8qc_me8q_build_opts* opts, void* stream);
/* Me8qIndex::SearchIVF (me8q_search.cpp:136-236): out rows of k ids /
 * distances, ascending; k <= 128. Host or device pointers. */
int e8qc_me8q_search(e8qc_me8q* idx, const float* queries, size_t nq, size_t k, size_t nprobe,
                     uint32_t* out_ids, float* out_dists, e8qc_stats* stats, void* stream);
/* Search with an explicit mode (an addition of this library):
 * E8QC_MODE_PRUNED is the reference's production search, the one its Python
 * Me8qIndex.search runs (SearchIVFFast / SearchIVFFastBatch,
 * src/index/me8q_fast.cpp:37-1090, python_bindings/me8q_bindings.cpp:97-160):
 * FastScan coarse plane, zero-parallel-residual bound with the build's
 * prune_alpha, run cascade against the running heap -- its prune decisions
 * in its own order, so its rows (the fast layout is built on first use,
 * about 1.4 B per coded block and 13 B per run per vector; uniform k and
 * nprobe; at most 16 coded runs and 512 coded blocks);
 * E8QC_MODE_BATCHED is e8qc_me8q_search (grouped exact scan, every candidate
 * scored with the estimator); E8QC_MODE_PRECISION generates candidates on the
 * INT8 tensor cores from an int8 plane of each vector's levels scaled by its
 * per-run coef (one scale per vector; built on first use, padded_dim bytes
 * per vector) and rescores each query's best max(32, 3k) (at most 128) with
 * the reference's estimator: returned distances are exact, recall against the
 * exact scan is measured. */
int e8qc_me8q_search_mode(e8qc_me8q* idx, const float* queries, size_t nq, size_t k, size_t nprobe, int mode,
                          uint32_t* out_ids, float* out_dists, e8qc_stats* stats, void* stream);
/* Serving form (an addition of this library): per-query k[i] <= k_max and
 * nprobe[i] (host arrays); output rows k_max wide, padded with UINT32_MAX /
 * +inf; mode as in e8qc_me8q_search_mode. */
int e8qc_me8q_search_ragged(e8qc_me8q* idx, const float* queries, size_t nq, const uint32_t* k,
                            const uint32_t* nprobe, size_t k_max, int mode, uint32_t* out_ids, float* out_dists,
                            void* stream);
/* Me8qIndex::Load (src/index/me8q_io.cpp:67-175): open an index file the
 * reference wrote with Me8qIndex::Save (ME8QIDXX) straight into a device index
 * on `device`: plan, rotator signs, centroids, ids, rows (codes, coef, h2) come
 * from the file, nothing is re-encoded. E8QC_EIO for an unreadable, foreign,
 * truncated or inconsistent file. */
int e8qc_me8q_load(int device, const char* path, e8qc_me8q** out);
/* Me8qIndex::Save (src/index/me8q_io.cpp:29-65): write the index as an
 * ME8QIDXX file the reference's Me8qIndex::Load reads (plan, padded
 * centroids, ids, offsets, rows packed as the reference packs them, rotator
 * seed and signs). E8QC_EIO when the file cannot be written. */
int e8qc_me8q_save(e8qc_me8q* idx, const char* path);
/* Me8qIndex::Estimate (me8q_measure.cpp:41-66); E8QC_ERANGE for an unknown id. */
int e8qc_me8q_estimate(e8qc_me8q* idx, const float* query, uint32_t id, float* out);
int e8qc_me8q_info(const e8qc_me8q* idx, e8qc_me8q_meta* out);
/* The plan (shared_plan, me8q.hpp:135): *count runs; up to cap (len, bits) written. */
int e8qc_me8q_plan(const e8qc_me8q* idx, size_t* lens, int* bits, size_t cap, size_t* count);
/* Global ids, cluster-major (n entries). */
int e8qc_me8q_get_ids(const e8qc_me8q* idx, uint32_t* out);
/* Per vector, cluster-major: digits n*padded_dim uint16 and branch
 * n*padded_dim/8 uint8 of every coded run (zeros in dropped runs), coef and
 * h2 n*ncoded floats (any may be NULL). */
int e8qc_me8q_export_codes(e8qc_me8q* idx, uint16_t* digits, uint8_t* branch, float* coef, float* h2);

/* ---- Autotuning and captured plans (no reference counterpart) ---- */
typedef struct e8qc_tuning {
    int schedule;      /* work-queue order: 0 longest list first, 1 list id order */
    int stages;        /* precision scan K-chunk ring depth: 4, 6 or 8 (6 in batched mode) */
    double best_ms;    /* one batch with the chosen setting (CUDA events) */
    double default_ms; /* one batch with the default setting (schedule 0, 6 stages) */
} e8qc_tuning;
/* Time the tunable settings of mode E8QC_MODE_BATCHED / E8QC_MODE_PRECISION
 * on nq synthetic queries (mixtures of the index's centroids) with k and
 * nprobe, and keep the fastest for this batch shape (power-of-two buckets of
 * nq and nprobe): later searches of that shape use it. Settings change the
 * order of work only; results are identical under every setting. */
int e8qc_e8q_autotune(e8qc_index* idx, int mode, size_t nq, size_t k, size_t nprobe, e8qc_tuning* out);

/* A captured search plan: for batch sizes 64, 128, ... up to max_queries it
 * autotunes (if asked), sizes its own workspace and captures the whole ragged
 * search (rotate, route, select, group, scan, merge / rescore) as one CUDA
 * graph. e8qc_plan_run pads a batch of nq <= max_queries queries (k[i] <=
 * k_max, nprobe[i] <= nprobe_max; host arrays) to the next captured size and
 * launches that graph on `stream`; queries and outputs may be host or device
 * pointers; out rows are k_max wide; it returns once the results are in the
 * outputs. One plan runs one batch at a time. The index must not be rebuilt
 * while a plan exists. */
typedef struct e8qc_plan e8qc_plan;
int e8qc_plan_create(e8qc_index* idx, int mode, size_t max_queries, size_t k_max, size_t nprobe_max, int autotune,
                     e8qc_plan** out);
/* The same over an ME8Q index, mode E8QC_MODE_BATCHED or E8QC_MODE_PRECISION. */
int e8qc_plan_create_me8q(e8qc_me8q* idx, int mode, size_t max_queries, size_t k_max, size_t nprobe_max,
                          int autotune, e8qc_plan** out);
int e8qc_plan_run(e8qc_plan* plan, const float* queries, size_t nq, const uint32_t* k, const uint32_t* nprobe,
                  uint32_t* out_ids, float* out_dists, void* stream);
int e8qc_plan_destroy(e8qc_plan* plan);

/* ---- Serving loop (no reference counterpart; the suggested
 * e8qc_serve_{start,submit,poll,stop} of the port plan) ----
 * A server owns a dispatcher and a completion thread over one built index.
 * Requests (nq queries sharing k and nprobe) are copied at submit and wait in
 * a FIFO until admitted: whenever one of `slots` batch slots is free, the
 * dispatcher takes pending requests in order while the batch stays within
 * max_batch_queries and its device-scratch estimate within memory_budget,
 * and enqueues the batch (H2D copy, rotate, route, grouped scan, D2H copy) on
 * the slot's own stream and workspace without waiting for it. Requests that
 * arrive while batches run join the next free slot (continuous batching);
 * batches on different slots overlap on the device. A query's result does
 * not depend on the batch it ran in. At start every slot runs, once, the
 * largest batch the budget admits at (max_k, max_nprobe), so its scratch is
 * allocated before the first request. The index must not be rebuilt or
 * destroyed while a server runs on it. */
typedef struct e8qc_server e8qc_server;
typedef struct e8qc_server_config {
    int mode;                 /* E8QC_MODE_BATCHED or E8QC_MODE_PRECISION */
    size_t max_batch_queries; /* queries per device batch (0 = 4096) */
    size_t max_k;             /* largest k a request may ask for (0 = 128) */
    size_t max_nprobe;        /* largest nprobe a request may ask for (0 = nlist) */
    size_t memory_budget;     /* device scratch bytes one batch may use (0 = 4 GiB) */
    int slots;                /* batches in flight (0 = 2) */
    int request_timeout_ms;   /* a request not admitted to a batch within this many ms of its
                                 submit fails with E8QC_ETIMEOUT (0 = no limit) */
} e8qc_server_config;
typedef struct e8qc_server_stats {
    uint64_t submitted, rejected, completed, failed, queries_completed, batches;
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> results ready, over completed requests */
    double qps;                             /* queries completed / (last completion - first submit) */
    double mean_batch_queries;
    uint64_t peak_batch_bytes;              /* largest admitted batch estimate */
    uint64_t canceled, expired;             /* requests canceled / expired before admission */
} e8qc_server_stats;
int e8qc_server_start(e8qc_index* idx, const e8qc_server_config* cfg, e8qc_server** out);
/* The serving loop over an ME8Q index (cfg->mode E8QC_MODE_BATCHED or
 * E8QC_MODE_PRECISION); submit / poll / stats / stop as above. */
int e8qc_server_start_me8q(e8qc_me8q* idx, const e8qc_server_config* cfg, e8qc_server** out);
/* Copy nq host queries (dim floats each) into a new request; *request_id
 * identifies it. E8QC_EINVAL for bad k / nprobe, E8QC_ENOMEM when the request
 * alone exceeds the memory budget or max_batch_queries, E8QC_ESTATE after stop. */
int e8qc_server_submit(e8qc_server* srv, const float* queries, size_t nq, size_t k, size_t nprobe,
                       uint64_t* request_id);
/* Wait up to timeout_ms (negative: forever) for a request. On completion
 * (*done = 1) the results (nq*k ids and distances, host buffers; either may be
 * NULL) are copied out and the request is released; the return value is the
 * request's own status (a failed batch reports its error). *done = 0 on
 * timeout. E8QC_ERANGE for an unknown or already collected id. */
int e8qc_server_poll(e8qc_server* srv, uint64_t request_id, int timeout_ms, uint32_t* out_ids, float* out_dists,
                     int* done);
/* Cancel a request. One still waiting for admission leaves the queue and
 * completes at once with E8QC_ECANCELED; one already in a batch on the device
 * completes with E8QC_ECANCELED when its batch ends (its rows are discarded);
 * one already complete keeps its results. The request is still collected with
 * e8qc_server_poll. E8QC_ERANGE for an unknown or already collected id. */
int e8qc_server_cancel(e8qc_server* srv, uint64_t request_id);
/* Counters and latency percentiles; reset = 1 clears them after the read. */
int e8qc_server_get_stats(e8qc_server* srv, int reset, e8qc_server_stats* out);
/* Stop accepting requests, finish the batches in flight, fail the requests
 * still pending (E8QC_ESTATE), join the threads and free the server. */
int e8qc_server_stop(e8qc_server* srv);

/* E8qIndex.probe_bound_w (python_bindings/e8q_bindings.cpp:182-233;
 * E8qIndex::ProbeBoundW, src/index/e8q_oracle.cpp:103-218): for m pairs, pair i
 * = query queries[qidx[i]] (nq x dim) against the stored vector ids[i] whose
 * raw build row is base_rows[i] (m x dim): the zero-parallel-residual bound's
 * normalised discrepancy (d_coarse^2 - d^2) / (r_q * Omega), every term in
 * double from the stored code, into out[m]. NaN where qidx[i] >= nq, the id
 * is not in the index, or the pair is degenerate. Host or device buffers. */
int e8qc_e8q_probe_bound_w(e8qc_index* idx, const float* queries, size_t nq, const float* base_rows,
                           const uint32_t* qidx, const uint32_t* ids, size_t m, double* out);

/* ---- Fault injection for callers' error paths (no reference counterpart) ----
 * Failures these calls provoke are made on the host or by a bounded device
 * wait; none of them faults, traps or hangs the GPU. */
/* The next `count` host allocations at the library's checked points --
 * creating an index (e8qc_e8q_create, e8qc_me8q_create) and taking in a
 * served request (e8qc_server_submit) -- fail as if the host were out of
 * memory: the call returns E8QC_ENOMEM and changes nothing. Process-wide;
 * count 0 clears it. */
int e8qc_debug_fail_host_allocs(int count);
/* The next `searches` plain searches of this index make their scan kernel
 * wait, bounded by wait_ms (1..10000), on a device barrier that nothing
 * completes -- the path a bulk copy that never lands would take. The wait
 * gives up, the kernel records it in the index's device error word, and the
 * search returns E8QC_ETIMEOUT; the index stays usable and later searches run
 * normally. searches 0 clears it. */
int e8qc_e8q_debug_inject_wait_timeout(e8qc_index* idx, int searches, uint32_t wait_ms);

#ifdef __cplusplus
}
#endif
#endif
