/* CPU restatement of the reference's ME8Q (mixed-rate E8Q) build and plain
 * search -- test infrastructure, the checker for the GPU path, never shipped.
 * Each function cites the reference file:line it follows. */
#ifndef ME8Q_ORACLE_H
#define ME8Q_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-dimension variance of the base rows (float mean, fp64 spread). */
void orc_me8q_variance(const float* base, size_t ld, size_t n, size_t dim, float* var);

/* SAQ DP bit allocation over 64-dim blocks; fills up to pd/64 runs and
 * returns their count. */
int orc_me8q_allocate(const float* var, size_t pd, float avg_bits, int max_bits, double extra_bits,
                      size_t* out_len, int* out_bits);

typedef struct orc_me8q_index orc_me8q_index;

orc_me8q_index* orc_me8q_build(const float* base, const float* centroids, const uint32_t* cluster_ids,
                               size_t n, size_t dim, size_t nlist, const size_t* plan_len,
                               const int* plan_bits, int nplan, uint64_t rot_seed, int drop_energy,
                               int threads);
void orc_me8q_free(orc_me8q_index* x);

/* Sizes: n, padded dim, number of coded runs. */
void orc_me8q_shape(const orc_me8q_index* x, size_t* n, size_t* pd, int* ncoded);

/* Codes of the vector in cluster-major position pos: digits (pd u16, 0 on
 * dropped dims), branch (pd/8 u8), coef / h2 per coded run. */
void orc_me8q_codes(const orc_me8q_index* x, size_t pos, uint16_t* digits, uint8_t* branch, float* coef,
                    float* h2);
/* Global ids in cluster-major order (n). */
void orc_me8q_ids(const orc_me8q_index* x, uint32_t* out);

float orc_me8q_estimate(const orc_me8q_index* x, const float* query, uint32_t id);
void orc_me8q_search(const orc_me8q_index* x, const float* queries, size_t nq, size_t k, size_t nprobe,
                     uint32_t* out_ids, float* out_dists, int threads);
/* The reference's production search (SearchIVFFast*, src/index/me8q_fast.cpp:
 * 37-1090, src/simd/me8q_prune_avx512.cpp:9-92): FastScan coarse plane,
 * zero-parallel-residual bound and run cascade against the live heap; alpha
 * is the build's prune_alpha. cand / surv (may be NULL): per query the scanned
 * candidates and the rows pushed to the heap. */
void orc_me8q_search_pruned(const orc_me8q_index* x, const float* queries, size_t nq, size_t k, size_t nprobe,
                            float alpha, uint32_t* out_ids, float* out_dists, uint64_t* cand, uint64_t* surv,
                            int threads);

#ifdef __cplusplus
}
#endif
#endif
