/* CPU oracle for the E8Q IVF search path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference e8qlib algorithm for this path
 * (every function cites the reference file:line it follows). Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it, and only as
 * the checker; the product (libe8qcuda.so and the e8qlib package) never links,
 * loads or calls anything here.
 *
 * Parity pins: tests/test_oracle_pins.py checks this restatement against the
 * reference compiled from its own sources (oracle/_ref, when present) and
 * against the committed golden vectors in tests/golden/ generated from it.
 */
#ifndef E8Q_ORACLE_H
#define E8Q_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_BITS 13

/* ---- codec constants ---------------------------------------------------- */
double orc_inv_normal_cdf(double p);
/* levels[d] = sigma_c * PhiInv(1/2 + (t+eta)/q), q = 2^bits entries. */
int orc_branch_levels(int bits, int branch, double* out);
double orc_fixed_scale(int bits);
/* table[br*stride + d] = (float)(level[br][d] / sqrt(padded_dim)),
 * stride = max(256, 2^bits); returns the table length 2*stride. */
int orc_refine_tables(int bits, int padded_dim, float* out);
void orc_scan_class_means(int bits, double w_cls[2]);
/* 1 when the merged four-class table of this rate alternates (the encoder's
 * single-search path), 0 when the encoder uses the four parity tables. */
int orc_merged_alternating(int bits);
/* Build the encoder's lookup tables for `bits` (they are created lazily and
 * are not safe to create from several threads at once: call this before a
 * parallel region that encodes). */
void orc_warm_tables(int bits);

/* ---- encoder ------------------------------------------------------------ */
/* n unit vectors (padded_dim floats each) -> digits[n][B][8], branch[n][B]. */
void orc_encode(const float* unit, size_t n, int padded_dim, int bits, double s,
                uint16_t* digits, uint8_t* branch);

/* ---- packing (the reference's on-disk/scan layout, one block) ----------- */
uint8_t orc_pack_coarse(const uint16_t digits[8], int branch, int bits);
void orc_pack_refine(const uint16_t digits[8], int branch, int bits, uint8_t* out);
void orc_decode_split(int bits, uint8_t rowa, const uint8_t* refine, uint16_t digits[8],
                      int* branch);

/* ---- rotator ------------------------------------------------------------ */
size_t orc_padded_dim(size_t dim);
size_t orc_sign_bytes(size_t dim);
void orc_rotator_signs(size_t dim, uint64_t seed, uint8_t* out);
void orc_rotate(size_t dim, const uint8_t* signs, const float* src, float* dst);

/* ---- index (plain path) ------------------------------------------------- */
typedef struct orc_e8q_index {
    size_t n, dim, padded_dim, nlist;
    int bits, blocks;
    uint8_t* signs;        /* 4*Dpad/8 */
    float* mean_rot;       /* Dpad */
    float* centroid_rot;   /* nlist*Dpad */
    float* cn2;            /* nlist */
    uint64_t* list_begin;  /* nlist+1 */
    uint32_t* ids;         /* n, cluster-major */
    uint16_t* digits;      /* n*B*8, cluster-major */
    uint8_t* branch;       /* n*B */
    float* g1;             /* n */
    float* h3;             /* n */
    float* tab;            /* 2*stride refine tables */
    int tab_stride;
    float* ortho;          /* n*3 scan-bank inputs per row: base, weight, perp */
} orc_e8q_index;

/* Restates E8qIndex::Build for everything the plain search reads. */
orc_e8q_index* orc_e8q_build(const float* base, const float* centroids,
                             const uint32_t* cluster_ids, size_t n, size_t dim,
                             size_t nlist, int bits, uint64_t seed, int threads);
void orc_e8q_free(orc_e8q_index* idx);

/* Rotated, mean-centred query (Dpad floats). */
void orc_e8q_prepare_query(const orc_e8q_index* idx, const float* q, float* rot_q);
/* fp64-accumulated exact score of cluster-major row `pos` (ExactScore). */
float orc_e8q_exact_score(const orc_e8q_index* idx, size_t pos, const float* rot_q);
/* Estimate(): fp32 d2 of the row's list + (d2+h3) - 2*g1*S. */
float orc_e8q_estimate(const orc_e8q_index* idx, const float* q, uint32_t id);
/* Route: keys (d2 bits << 32 | cid) of the nprobe nearest lists, ascending. */
void orc_e8q_route(const orc_e8q_index* idx, const float* rot_q, size_t nprobe,
                   uint32_t* probe_ids, float* probe_d2);
/* Plain (unpruned) search of nq queries: ids/dists [nq][k]; missing slots are
 * UINT32_MAX / +inf. threads: OpenMP threads over queries. */
void orc_e8q_search(const orc_e8q_index* idx, const float* queries, size_t nq, size_t k,
                    size_t nprobe, uint32_t* out_ids, float* out_dists, int threads);

/* ---- pruned production path -------------------------------------------
 * The reference's shipped search: a coarse pass prices one rowA byte per
 * block against a u8 LUT, a zero-parallel-residual lower bound dlo rejects
 * rows that cannot beat the current k-th distance, and the survivors are
 * refined exactly. */

/* PhiInv (Newton on Phi) and OrthoQuantile: src/index/e8q_internal.hpp:75-107. */
double orc_phi_inv(double p);
float orc_ortho_quantile(double alpha, size_t k_eff);
/* One 128-byte batch header from its rows' bank inputs (WriteOrthoBanks,
 * src/index/e8q_build.cpp:31-80). */
void orc_ortho_header(const float* base, const float* weight, const float* perp, size_t cnt,
                      uint8_t* hdr);
/* Headers of every 32-row batch, lists in order (128 B each); returns the
 * batch count (out may be NULL to count). */
size_t orc_e8q_banks(const orc_e8q_index* idx, uint8_t* out);
/* rowA byte of cluster-major row `pos`, block blk (PackCoarseRow). */
uint8_t orc_e8q_rowa(const orc_e8q_index* idx, size_t pos, int blk);
/* PrepareQuery (src/index/e8q_search.cpp:20-73): the u8 coarse LUT, 32 bytes
 * per block ([0,16) prices the low nibble = digits 4..7, [16,32) the high
 * nibble = digits 0..3) and scal = {delta_c, base_c, lut_err, score_max}. */
void orc_e8q_prepare_lut(int bits, int blocks, const float* rot_q, uint8_t* lut, float* scal);
/* Coarse sum of the row's rowA bytes against the LUT (AccumulateCoarseHi,
 * src/simd/scan_kernels_generic.cpp:12-35); pos == (size_t)-1 prices an
 * all-zero padding row. */
int32_t orc_e8q_coarse(const orc_e8q_index* idx, size_t pos, const uint8_t* lut);
/* The refine arithmetic of the shipped search (RefineRowsAvx512,
 * src/simd/e8q_search_avx512.cpp:118-347): eight fp32 dimension lanes, even
 * and odd blocks in separate fused chains, then HsumPs. */
float orc_e8q_refine_score(const orc_e8q_index* idx, size_t pos, const float* rot_q);
/* The shipped sequential search (E8qIndex::Search, e8q_search.cpp:215-293,
 * with ScanClusterAvx512 and CollectLanes): lists in probe order, batches of
 * 32 in order, survivors refined every 32 staged rows and at the end of each
 * list. banks: the 128-byte headers (orc_e8q_banks order), NULL for this
 * oracle's own. cand/surv (may be NULL): per query rows scanned / refined. */
void orc_e8q_search_pruned(const orc_e8q_index* idx, const uint8_t* banks, float alpha,
                           int disable_prune, const float* queries, size_t nq, size_t k,
                           size_t nprobe, uint32_t* out_ids, float* out_dists, uint64_t* cand,
                           uint64_t* surv, int threads);

/* ProbeBoundW (src/index/e8q_oracle.cpp:103-218): for the stored vector `id`
 * whose raw build input is base_row, the normalised discrepancy
 * (d_coarse^2 - d^2) / (r_q * Omega) of the zero-parallel-residual bound,
 * every term recomputed in double from the stored codes; NaN for a
 * degenerate pair or an id not in the index. */
double orc_e8q_probe_bound_w(const orc_e8q_index* idx, const float* query, const float* base_row, uint32_t id);

#ifdef __cplusplus
}
#endif
#endif
