/* CPU restatement of the reference's ME8Q build and plain search (test
 * infrastructure: the checker for the GPU path; nothing shipped calls it).
 *
 * Multiply-adds the reference's GCC build contracts (C++ default
 * -ffp-contract=fast with an FMA -march) are spelled out with fma()/fmaf();
 * this file is compiled with -ffp-contract=off so no others appear. */
#include "me8q_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "e8q_oracle.h"

#define SEG_DIM 64   /* include/e8qlib/quantization/me8q_plan.hpp:20 kSegDim */
#define MAX_BITS 13  /* :21 kMaxBits */
#define FACTOR_BITS 64 /* :22 kFactorBits */

/* detail::DatasetVariance, src/index/me8q_common.cpp:11-35: float mean
 * accumulated row by row, fp64 spread, float result. */
void orc_me8q_variance(const float* base, size_t ld, size_t n, size_t dim, float* var) {
    float* mean = (float*)calloc(dim, sizeof(float));
    double* tmp = (double*)calloc(dim, sizeof(double));
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < dim; ++j) mean[j] += base[i * ld + j];
    for (size_t j = 0; j < dim; ++j) mean[j] /= (float)n;
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < dim; ++j) {
            const double d = (double)base[i * ld + j] - mean[j];
            tmp[j] = fma(d, d, tmp[j]);
        }
    for (size_t j = 0; j < dim; ++j) var[j] = (float)(tmp[j] / (double)n);
    free(mean);
    free(tmp);
}

/* Allocate (SAQ's DP), src/quantization/me8q_plan.cpp:47-167: runs of whole
 * 64-dim blocks at 1..max_bits, a trailing 0-bit run priced at its variance,
 * budget in units of 64 bits (each run costs b*j + 1 units), at most
 * nblocks/2 runs for avg_bits >= 2, and SAQ's acceptance rule (cur*1.01 <
 * best). Cost of a run: sum var / 2^b (BuildCostTable :16-40). */
int orc_me8q_allocate(const float* var, size_t pd, float avg_bits, int max_bits, double extra_bits,
                      size_t* out_len, int* out_bits) {
    const size_t nb = pd / SEG_DIM;
    const double budget = (double)avg_bits * (double)pd + extra_bits + (double)FACTOR_BITS;
    const size_t tot_bits = budget > 0.0 ? (size_t)budget : 0;
    const size_t units = tot_bits / SEG_DIM;
    const size_t max_segs = avg_bits < 2.0F ? nb : nb / 2;
    double* p1 = (double*)calloc(nb + 1, sizeof(double));
    for (size_t b = 0; b < nb; ++b) {
        double s = 0.0;
        for (size_t k = 0; k < SEG_DIM; ++k) s += (double)var[b * SEG_DIM + k];
        p1[b + 1] = p1[b] + s;
    }
    const double total = p1[nb];
    const size_t span_i = nb + 1, span_t = units + 1;
    const size_t layer = span_i * span_t;
    double* f = (double*)malloc(sizeof(double) * (max_segs + 1) * layer);
    uint32_t* pred = (uint32_t*)calloc((max_segs + 1) * layer, sizeof(uint32_t));
    for (size_t i = 0; i < (max_segs + 1) * layer; ++i) f[i] = DBL_MAX;
#define AT(ns, i, t) (((ns) * span_i + (i)) * span_t + (t))
    f[AT(0, 0, 0)] = 0.0;
    double best = DBL_MAX;
    size_t ans_ns = 0, ans_t = 0;
    for (size_t ns = 0; ns <= max_segs; ++ns)
        for (size_t i = 0; i <= nb; ++i)
            for (size_t t = 0; t <= units; ++t) {
                const double cur = f[AT(ns, i, t)];
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
                        const size_t t2 = t + (size_t)b * j + 1;
                        if (t2 > units) break;
                        const double v = cur + vsum / (double)((int64_t)1 << b);
                        const size_t to = AT(ns + 1, i + j, t2);
                        if (v < f[to]) {
                            f[to] = v;
                            pred[to] = (uint32_t)((i << 4) | (size_t)b);
                        }
                    }
                }
                const double rest = total - p1[i];
                const size_t to = AT(ns + 1, nb, t);
                if (cur + rest < f[to]) {
                    f[to] = cur + rest;
                    pred[to] = (uint32_t)(i << 4);
                }
            }
    int nrun = 0;
    if (best >= DBL_MAX) {
        /* no feasible plan: the single all-dropped run (:133-147) */
        out_len[0] = pd;
        out_bits[0] = 0;
        nrun = 1;
    } else {
        size_t lens[64];
        int bits[64];
        size_t ns = ans_ns, i = nb, t = ans_t;
        while (i > 0) {
            const uint32_t p = pred[AT(ns, i, t)];
            const size_t prev_i = p >> 4;
            const int b = (int)(p & 0xF);
            lens[nrun] = (i - prev_i) * SEG_DIM;
            bits[nrun] = b;
            ++nrun;
            ns--;
            if (b != 0) t -= (size_t)b * (i - prev_i) + 1;
            i = prev_i;
        }
        for (int r = 0; r < nrun; ++r) {
            out_len[r] = lens[nrun - 1 - r];
            out_bits[r] = bits[nrun - 1 - r];
        }
    }
#undef AT
    free(p1);
    free(f);
    free(pred);
    return nrun;
}

typedef struct {
    size_t off, len;
    int bits;
    uint8_t* signs; /* the run's rotator (coded runs only) */
} orc_run;

struct orc_me8q_index {
    size_t n, dim, pd, nlist, route_dim;
    int nplan, ncoded;
    orc_run* runs; /* all plan runs, in order */
    int drop_energy;
    float* centroids;   /* nlist x pd, padded */
    float* cent_rot;    /* per-run rotated centroids, dropped tail zero */
    float* cn2;         /* ||cent_rot||^2 */
    uint64_t* list_begin;
    uint32_t* ids;      /* cluster-major */
    uint16_t* digits;   /* cluster-major n x pd */
    uint8_t* branch;    /* n x pd/8 */
    float* coef;        /* n x ncoded */
    float* h2;
    double lev[MAX_BITS + 1][2][1 << MAX_BITS]; /* raw levels (float-rounded), SegmentCodec ctor :13-33 */
    float levf[MAX_BITS + 1][2][1 << MAX_BITS];
};

/* Per-run rotators with golden-ratio seed steps: BuildRunRotators,
 * src/index/me8q_build.cpp:29-40. */
static void make_runs(orc_me8q_index* x, const size_t* plan_len, const int* plan_bits, int nplan, uint64_t seed) {
    x->runs = (orc_run*)calloc((size_t)nplan, sizeof(orc_run));
    x->nplan = nplan;
    x->ncoded = 0;
    uint64_t s = seed;
    size_t off = 0;
    for (int r = 0; r < nplan; ++r) {
        x->runs[r].off = off;
        x->runs[r].len = plan_len[r];
        x->runs[r].bits = plan_bits[r];
        if (plan_bits[r] != 0) {
            s += 0x9E3779B97F4A7C15ULL;
            x->runs[r].signs = (uint8_t*)malloc(orc_sign_bytes(plan_len[r]));
            orc_rotator_signs(plan_len[r], s, x->runs[r].signs);
            x->ncoded++;
        }
        off += plan_len[r];
    }
}

/* PrepareRotatedQuery / PrepareCentroidsRotated, src/index/me8q_search.cpp:31-72:
 * one rotation per coded run, dropped tail left as the caller set it. */
static void rotate_runs(const orc_me8q_index* x, const float* src, float* dst) {
    for (int r = 0; r < x->nplan; ++r)
        if (x->runs[r].bits != 0) orc_rotate(x->runs[r].len, x->runs[r].signs, src + x->runs[r].off, dst + x->runs[r].off);
}

orc_me8q_index* orc_me8q_build(const float* base, const float* centroids, const uint32_t* cluster_ids,
                               size_t n, size_t dim, size_t nlist, const size_t* plan_len,
                               const int* plan_bits, int nplan, uint64_t rot_seed, int drop_energy,
                               int threads) {
    orc_me8q_index* x = (orc_me8q_index*)calloc(1, sizeof(orc_me8q_index));
    x->n = n;
    x->dim = dim;
    x->pd = orc_padded_dim(dim);
    x->nlist = nlist;
    x->drop_energy = drop_energy;
    const size_t pd = x->pd;
    for (int b = 1; b <= MAX_BITS; ++b)
        for (int br = 0; br < 2; ++br) {
            orc_branch_levels(b, br, x->lev[b][br]);
            for (int d = 0; d < (1 << b); ++d) {
                x->levf[b][br][d] = (float)x->lev[b][br][d];
                x->lev[b][br][d] = (double)x->levf[b][br][d];
            }
        }
    make_runs(x, plan_len, plan_bits, nplan, rot_seed);
    for (int r = 0; r < nplan; ++r)
        if (plan_bits[r] != 0) orc_warm_tables(plan_bits[r]); /* before the threads share them */
    /* padded centroids, per-run rotation, norms (CentroidNorm2,
     * include/e8qlib/index/ivf_common.hpp:43-54) */
    x->centroids = (float*)calloc(nlist * pd, sizeof(float));
    x->cent_rot = (float*)calloc(nlist * pd, sizeof(float));
    x->cn2 = (float*)malloc(sizeof(float) * nlist);
    for (size_t c = 0; c < nlist; ++c) {
        memcpy(x->centroids + c * pd, centroids + c * dim, dim * sizeof(float));
        rotate_runs(x, x->centroids + c * pd, x->cent_rot + c * pd);
        double s = 0.0;
        for (size_t d = 0; d < pd; ++d)
            s = fma((double)x->cent_rot[c * pd + d], (double)x->cent_rot[c * pd + d], s);
        x->cn2[c] = (float)s;
    }
    x->route_dim = pd;
    for (int r = nplan - 1; r >= 0 && plan_bits[r] == 0; --r) x->route_dim -= plan_len[r];
    /* lists (ivf::BuildLists: stable by cluster) */
    x->list_begin = (uint64_t*)calloc(nlist + 1, sizeof(uint64_t));
    for (size_t i = 0; i < n; ++i) x->list_begin[cluster_ids[i] + 1]++;
    for (size_t c = 0; c < nlist; ++c) x->list_begin[c + 1] += x->list_begin[c];
    x->ids = (uint32_t*)malloc(sizeof(uint32_t) * n);
    size_t* fill = (size_t*)calloc(nlist, sizeof(size_t));
    size_t* pos_of = (size_t*)malloc(sizeof(size_t) * n);
    for (size_t i = 0; i < n; ++i) {
        const size_t c = cluster_ids[i];
        const size_t p = x->list_begin[c] + fill[c]++;
        x->ids[p] = (uint32_t)i;
        pos_of[i] = p;
    }
    free(fill);
    x->digits = (uint16_t*)calloc(n * pd, sizeof(uint16_t));
    x->branch = (uint8_t*)calloc(n * (pd / 8), 1);
    x->coef = (float*)calloc(n * (size_t)(x->ncoded > 0 ? x->ncoded : 1), sizeof(float));
    x->h2 = (float*)calloc(n * (size_t)(x->ncoded > 0 ? x->ncoded : 1), sizeof(float));
    /* encode, src/index/me8q_build.cpp:203-309 */
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        float* resid = (float*)malloc(sizeof(float) * pd);
        float* rrot = (float*)malloc(sizeof(float) * pd);
        float* unit = (float*)malloc(sizeof(float) * pd);
#pragma omp for schedule(dynamic, 64)
        for (long long ri = 0; ri < (long long)n; ++ri) {
            const size_t row = (size_t)ri;
            const size_t c = cluster_ids[row];
            const size_t p = pos_of[row];
            memset(resid, 0, sizeof(float) * pd);
            memset(rrot, 0, sizeof(float) * pd);
            for (size_t j = 0; j < dim; ++j) resid[j] = base[row * dim + j] - x->centroids[c * pd + j];
            rotate_runs(x, resid, rrot);
            double drop_n2 = 0.0;
            if (drop_energy)
                for (int r = 0; r < nplan; ++r)
                    if (x->runs[r].bits == 0)
                        for (size_t j = 0; j < x->runs[r].len; ++j) {
                            const double v = (double)resid[x->runs[r].off + j];
                            drop_n2 = fma(v, v, drop_n2);
                        }
            int slot = 0;
            for (int r = 0; r < nplan; ++r) {
                const orc_run* run = &x->runs[r];
                if (run->bits == 0) continue;
                const float* rr = rrot + run->off;
                const int len = (int)run->len, bits = run->bits;
                double norm2 = 0.0;
                for (int j = 0; j < len; ++j) norm2 = fma((double)rr[j], (double)rr[j], norm2);
                const double norm = sqrt(norm2);
                uint16_t* dg = x->digits + p * pd + run->off;
                uint8_t* br = x->branch + p * (pd / 8) + run->off / 8;
                if (norm > 0.0) {
                    /* SegmentCodec::EncodeInto, src/quantization/me8q_codec.cpp:69-97 */
                    const double inv = 1.0 / norm;
                    for (int j = 0; j < len; ++j) unit[j] = (float)((double)rr[j] * inv);
                    orc_encode(unit, 1, len, bits, orc_fixed_scale(bits), dg, br);
                }
                /* ScoreVectorCode fits, me8q_codec.cpp:149-167 */
                double dot_r = 0.0, dot_c = 0.0;
                const float* cr = x->cent_rot + c * pd + run->off;
                for (int blk = 0; blk < len / 8; ++blk) {
                    const float* lv = x->levf[bits][br[blk] ? 1 : 0];
                    for (int i = 0; i < 8; ++i) {
                        const double l = (double)lv[dg[blk * 8 + i]];
                        dot_r = fma((double)rr[blk * 8 + i], l, dot_r);
                        dot_c = fma((double)cr[blk * 8 + i], l, dot_c);
                    }
                }
                double coef = dot_r > 1e-12 ? norm2 / dot_r : 0.0;
                if (!isfinite(coef)) coef = 0.0;
                double h2 = fma(2.0 * coef, dot_c, norm2);
                if (slot == x->ncoded - 1) h2 += drop_n2;
                x->coef[p * (size_t)x->ncoded + (size_t)slot] = (float)coef;
                x->h2[p * (size_t)x->ncoded + (size_t)slot] = (float)(isfinite(h2) ? h2 : 0.0);
                ++slot;
            }
        }
        free(resid);
        free(rrot);
        free(unit);
    }
    free(pos_of);
    return x;
}

void orc_me8q_free(orc_me8q_index* x) {
    if (!x) return;
    for (int r = 0; r < x->nplan; ++r) free(x->runs[r].signs);
    free(x->runs);
    free(x->centroids);
    free(x->cent_rot);
    free(x->cn2);
    free(x->list_begin);
    free(x->ids);
    free(x->digits);
    free(x->branch);
    free(x->coef);
    free(x->h2);
    free(x);
}

void orc_me8q_shape(const orc_me8q_index* x, size_t* n, size_t* pd, int* ncoded) {
    *n = x->n;
    *pd = x->pd;
    *ncoded = x->ncoded;
}

void orc_me8q_codes(const orc_me8q_index* x, size_t pos, uint16_t* digits, uint8_t* branch, float* coef, float* h2) {
    if (digits) memcpy(digits, x->digits + pos * x->pd, x->pd * sizeof(uint16_t));
    if (branch) memcpy(branch, x->branch + pos * (x->pd / 8), x->pd / 8);
    if (coef) memcpy(coef, x->coef + pos * (size_t)x->ncoded, (size_t)x->ncoded * sizeof(float));
    if (h2) memcpy(h2, x->h2 + pos * (size_t)x->ncoded, (size_t)x->ncoded * sizeof(float));
}

void orc_me8q_ids(const orc_me8q_index* x, uint32_t* out) { memcpy(out, x->ids, x->n * sizeof(uint32_t)); }

/* EstimateRow with the scalar segment score (ScoreFastGeneric,
 * src/simd/me8q_score_generic.cpp:37-64; EstimateRow, me8q_search.cpp:74-95):
 * d2 + sum_s (h2_s - 2 coef_s S_s), S_s = sum q_rot * level (fp32). */
static double estimate_row(const orc_me8q_index* x, size_t pos, double d2, const float* rq) {
    double acc = d2;
    int slot = 0;
    for (int r = 0; r < x->nplan; ++r) {
        const orc_run* run = &x->runs[r];
        if (run->bits == 0) continue;
        const double coef = x->coef[pos * (size_t)x->ncoded + (size_t)slot];
        const double h2 = x->h2[pos * (size_t)x->ncoded + (size_t)slot];
        ++slot;
        if (coef == 0.0) {
            acc += h2;
            continue;
        }
        const uint16_t* dg = x->digits + pos * x->pd + run->off;
        const uint8_t* br = x->branch + pos * (x->pd / 8) + run->off / 8;
        const float* q = rq + run->off;
        float s = 0.0F;
        for (size_t blk = 0; blk < run->len / 8; ++blk) {
            const float* lv = x->levf[run->bits][br[blk] ? 1 : 0];
            for (int i = 0; i < 8; ++i) s = fmaf(q[blk * 8 + i], lv[dg[blk * 8 + i]], s);
        }
        acc += fma(-2.0 * coef, (double)s, h2);
    }
    return acc;
}

static void prepare_query(const orc_me8q_index* x, const float* q, float* qpad, float* rq) {
    memset(qpad, 0, sizeof(float) * x->pd);
    memcpy(qpad, q, sizeof(float) * x->dim);
    memset(rq, 0, sizeof(float) * x->pd);
    rotate_runs(x, qpad, rq);
}

/* Estimate, src/index/me8q_measure.cpp:41-66: fp64 ||q - c||^2 in the
 * unrotated padded domain. */
float orc_me8q_estimate(const orc_me8q_index* x, const float* query, uint32_t id) {
    float* qpad = (float*)malloc(sizeof(float) * x->pd);
    float* rq = (float*)malloc(sizeof(float) * x->pd);
    prepare_query(x, query, qpad, rq);
    size_t pos = 0, c = 0;
    for (; pos < x->n; ++pos)
        if (x->ids[pos] == id) break;
    while (x->list_begin[c + 1] <= pos) ++c;
    double d2 = 0.0;
    for (size_t j = 0; j < x->pd; ++j) {
        const double d = (double)qpad[j] - x->centroids[c * x->pd + j];
        d2 = fma(d, d, d2);
    }
    const float out = (float)estimate_row(x, pos, d2, rq);
    free(qpad);
    free(rq);
    return out;
}

static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* RouteL2 over the coded prefix (QueryNorm2 + GEMV in fp64, key =
 * (bits(d2) << 32) | c, ivf_route.cpp:9-27, kernels_generic.cpp:5-33): d2 of
 * every list and the keys sorted ascending. */
static void route_query(const orc_me8q_index* x, const float* rq, float* d2, uint64_t* keys) {
    double qs = 0.0;
    for (size_t d = 0; d < x->route_dim; ++d) qs = fma((double)rq[d], (double)rq[d], qs);
    const float qn2 = (float)qs;
    for (size_t c = 0; c < x->nlist; ++c) {
        double dot = 0.0;
        const float* cc = x->cent_rot + c * x->pd;
        for (size_t d = 0; d < x->route_dim; ++d) dot = fma((double)rq[d], (double)cc[d], dot);
        float v = fmaf(-2.0F, (float)dot, qn2 + x->cn2[c]);
        if (v < 0.0F) v = 0.0F;
        d2[c] = v;
        uint32_t bv;
        memcpy(&bv, &v, 4);
        keys[c] = ((uint64_t)bv << 32) | (uint64_t)c;
    }
    qsort(keys, x->nlist, sizeof(uint64_t), cmp_u64);
}

/* SearchIVF, src/index/me8q_search.cpp:136-236: RouteL2 over the coded
 * prefix (QueryNorm2 + GEMV in fp64, key = (bits(d2) << 32) | c,
 * ivf_route.cpp:9-27, kernels_generic.cpp:5-33), every row of every probed
 * list estimated, sorted insert by distance (PushCandidate :121-134: an
 * equal distance goes before the earlier ones). */
void orc_me8q_search(const orc_me8q_index* x, const float* queries, size_t nq, size_t k, size_t nprobe,
                     uint32_t* out_ids, float* out_dists, int threads) {
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        float* qpad = (float*)malloc(sizeof(float) * x->pd);
        float* rq = (float*)malloc(sizeof(float) * x->pd);
        uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * x->nlist);
        float* d2 = (float*)malloc(sizeof(float) * x->nlist);
        float* hd = (float*)malloc(sizeof(float) * (k + 1));
        uint32_t* hi = (uint32_t*)malloc(sizeof(uint32_t) * (k + 1));
#pragma omp for schedule(dynamic, 1)
        for (long long qi = 0; qi < (long long)nq; ++qi) {
            prepare_query(x, queries + (size_t)qi * x->dim, qpad, rq);
            route_query(x, rq, d2, keys);
            const size_t take = nprobe < x->nlist ? nprobe : x->nlist;
            size_t cnt = 0;
            for (size_t p = 0; p < take; ++p) {
                const size_t c = (uint32_t)keys[p];
                for (size_t pos = x->list_begin[c]; pos < x->list_begin[c + 1]; ++pos) {
                    const float dist = (float)estimate_row(x, pos, (double)d2[c], rq);
                    if (cnt >= k && !(dist < hd[cnt - 1])) continue;
                    if (cnt >= k) --cnt;
                    size_t at = 0;
                    while (at < cnt && hd[at] < dist) ++at;
                    memmove(hd + at + 1, hd + at, (cnt - at) * sizeof(float));
                    memmove(hi + at + 1, hi + at, (cnt - at) * sizeof(uint32_t));
                    hd[at] = dist;
                    hi[at] = x->ids[pos];
                    ++cnt;
                }
            }
            for (size_t j = 0; j < k; ++j) {
                out_ids[(size_t)qi * k + j] = j < cnt ? hi[j] : 0xFFFFFFFFu;
                if (out_dists) out_dists[(size_t)qi * k + j] = j < cnt ? hd[j] : INFINITY;
            }
        }
        free(qpad);
        free(rq);
        free(keys);
        free(d2);
        free(hd);
        free(hi);
    }
}

/* ===== the production FastScan search (Me8qIndex::SearchIVFFast*) ========
 * BuildFastLayout, src/index/me8q_fast.cpp:37-307: per coded run r of a
 * vector the top-bit plane (rate >= 2: each digit's top bit; rate 1: the
 * sign bits of dims 0..6 and the branch in bit 0), the zero-parallel-residual
 * fit on the scan basis w = pbar[top bit] (gain, vpc, perp) and per batch of
 * 32 rows the u8 banks (base floor, weight nearest, perp ceil) with their
 * scales. The layout is global (one plan), so the per-run fields below are
 * shared by every list. */
typedef struct {
    int nrun;
    int* roff;      /* dim offset of coded run r */
    int* rlen;
    int* rbits;
    int* rslot;     /* index among the vector's (coef, h2) */
    int* blk0;      /* first plane column of run r */
    int cols;       /* plane columns (blocks) per vector */
    uint8_t* plane; /* n x cols, cluster-major */
    float* gain;    /* n x nrun */
    float* vpc;
    uint8_t* bank;  /* per (list batch, run): base[32] weight[32] perp[32] */
    float* scl;     /* per (list batch, run): 6 scales */
    size_t* batch0; /* first batch of list c */
    double* rc_n2;  /* nlist x nrun */
    float pbar[MAX_BITS + 1][2];
} orc_fast;

/* ClassModelOf, src/quantization/me8q_codec.cpp:235-262 (pbar only). */
static void class_pbar(const orc_me8q_index* x, int bits, float pbar[2]) {
    const int q = 1 << bits, half = q >> 1;
    for (int c = 0; c < 2; ++c) {
        double sum = 0.0;
        for (int br = 0; br < 2; ++br)
            for (int d = c * half; d < (c + 1) * half; ++d) sum += (double)x->levf[bits][br][d];
        pbar[c] = (float)(sum / (double)(2 * half));
    }
}

static int plane_top(const orc_me8q_index* x, size_t pos, int bits, size_t dim) {
    const int d = x->digits[pos * x->pd + dim];
    if (bits == 1 && (dim & 7) == 7) return x->branch[pos * (x->pd / 8) + dim / 8] & 1;
    return (d >> (bits - 1)) & 1;
}

static void fast_free(orc_fast* f) {
    free(f->roff);
    free(f->rlen);
    free(f->rbits);
    free(f->rslot);
    free(f->blk0);
    free(f->plane);
    free(f->gain);
    free(f->vpc);
    free(f->bank);
    free(f->scl);
    free(f->batch0);
    free(f->rc_n2);
}

/* The multiply-adds the reference's compiler fuses (GCC, FMA on, contract
 * fast) are spelled as fma() here. */
static void fast_build(const orc_me8q_index* x, orc_fast* f) {
    memset(f, 0, sizeof(*f));
    f->nrun = x->ncoded;
    const int nr = f->nrun;
    f->roff = (int*)calloc((size_t)nr + 1, sizeof(int));
    f->rlen = (int*)calloc((size_t)nr + 1, sizeof(int));
    f->rbits = (int*)calloc((size_t)nr + 1, sizeof(int));
    f->rslot = (int*)calloc((size_t)nr + 1, sizeof(int));
    f->blk0 = (int*)calloc((size_t)nr + 1, sizeof(int));
    int r = 0;
    for (int p = 0; p < x->nplan; ++p) {
        if (x->runs[p].bits == 0) continue;
        f->roff[r] = (int)x->runs[p].off;
        f->rlen[r] = (int)x->runs[p].len;
        f->rbits[r] = x->runs[p].bits;
        f->rslot[r] = r;
        f->blk0[r] = f->cols;
        f->cols += f->rlen[r] / 8;
        ++r;
    }
    for (int b = 1; b <= MAX_BITS; ++b) class_pbar(x, b, f->pbar[b]);
    const size_t n = x->n, cols = (size_t)f->cols;
    f->plane = (uint8_t*)calloc(n * cols + 1, 1);
    f->gain = (float*)calloc(n * (size_t)nr + 1, sizeof(float));
    f->vpc = (float*)calloc(n * (size_t)nr + 1, sizeof(float));
    f->batch0 = (size_t*)calloc(x->nlist + 1, sizeof(size_t));
    for (size_t c = 0; c < x->nlist; ++c)
        f->batch0[c + 1] = f->batch0[c] + (size_t)((x->list_begin[c + 1] - x->list_begin[c] + 31) / 32);
    const size_t nb = f->batch0[x->nlist];
    f->bank = (uint8_t*)calloc(nb * (size_t)nr * 96 + 1, 1);
    f->scl = (float*)calloc(nb * (size_t)nr * 6 + 1, sizeof(float));
    f->rc_n2 = (double*)calloc(x->nlist * (size_t)nr + 1, sizeof(double));
    float* perp = (float*)calloc(n * (size_t)nr + 1, sizeof(float));
    for (size_t c = 0; c < x->nlist; ++c) {
        for (int rr = 0; rr < nr; ++rr) {
            const float* rc = x->cent_rot + c * x->pd + f->roff[rr];
            double a = 0.0;
            for (int t = 0; t < f->rlen[rr]; ++t) a = fma((double)rc[t], (double)rc[t], a);
            f->rc_n2[c * (size_t)nr + (size_t)rr] = a;
        }
        for (size_t pos = x->list_begin[c]; pos < x->list_begin[c + 1]; ++pos) {
            for (int rr = 0; rr < nr; ++rr) {
                const int bits = f->rbits[rr], len = f->rlen[rr], nblk = len / 8;
                for (int blk = 0; blk < nblk; ++blk) {
                    uint8_t byte = 0;
                    for (int t = 0; t < 8; ++t)
                        if (plane_top(x, pos, bits, (size_t)(f->roff[rr] + blk * 8 + t)))
                            byte = (uint8_t)(byte | (1u << (7 - t)));
                    f->plane[pos * cols + (size_t)(f->blk0[rr] + blk)] = byte;
                }
                /* the fit, me8q_fast.cpp:140-230 */
                double dot_ew = 0.0, n2_w = 0.0, n2_e = 0.0, dot_ce = 0.0, dot_cw = 0.0;
                const float* rc = x->cent_rot + c * x->pd + f->roff[rr];
                for (int blk = 0; blk < nblk; ++blk) {
                    const int br = x->branch[pos * (x->pd / 8) + (size_t)(f->roff[rr] / 8 + blk)] ? 1 : 0;
                    for (int t = 0; t < 8; ++t) {
                        const int d = x->digits[pos * x->pd + (size_t)(f->roff[rr] + blk * 8 + t)];
                        const double ve = (double)x->levf[bits][br][d];
                        const double wc = (bits == 1 && t == 7) ? 0.0 : (double)f->pbar[bits][d >> (bits - 1)];
                        const double cv = (double)rc[blk * 8 + t];
                        dot_ew = fma(ve, wc, dot_ew);
                        n2_w = fma(wc, wc, n2_w);
                        n2_e = fma(ve, ve, n2_e);
                        dot_ce = fma(cv, ve, dot_ce);
                        dot_cw = fma(cv, wc, dot_cw);
                    }
                }
                const double coef = (double)x->coef[pos * (size_t)x->ncoded + (size_t)f->rslot[rr]];
                const double h2 = (double)x->h2[pos * (size_t)x->ncoded + (size_t)f->rslot[rr]];
                double rn2 = fma(-(2.0 * coef), dot_ce, h2);
                if (rn2 < 0.0) rn2 = 0.0;
                const double rn = sqrt(rn2);
                const double sqrt_lm1 = sqrt((double)(len - 1 > 1 ? len - 1 : 1));
                const double abs_c = fabs(coef);
                const size_t o = pos * (size_t)nr + (size_t)rr;
                if (n2_e > 1e-30 && abs_c > 1e-30) {
                    const double ve_norm = sqrt(n2_e);
                    const double n2_w_safe = n2_w > 1e-30 ? n2_w : 1e-30;
                    const double dot_uw = dot_ew / ve_norm;
                    const double uw_eps = 1e-12 * sqrt(n2_w_safe);
                    double wx, norm_rx;
                    if (fabs(dot_uw) > uw_eps) {
                        wx = 2.0 * rn / dot_uw;
                        const double rx2 = fma(-(4.0 * coef * wx), dot_ew, fma(4.0 * coef * coef, n2_e, wx * wx * n2_w));
                        norm_rx = sqrt(rx2 > 0.0 ? rx2 : 0.0);
                    } else {
                        const double gamma = dot_ew / n2_w_safe;
                        wx = 2.0 * coef * gamma;
                        double vp2 = fma(-(gamma * gamma), n2_w, n2_e);
                        if (vp2 < 0.0) vp2 = 0.0;
                        norm_rx = 2.0 * abs_c * sqrt(vp2);
                    }
                    f->gain[o] = (float)(wx / (2.0 * abs_c));
                    f->vpc[o] = (float)(fma(-wx, dot_cw, h2 - rn2) / (2.0 * abs_c));
                    perp[o] = (float)((norm_rx / sqrt_lm1) / (2.0 * abs_c));
                } else if (n2_w > 1e-30) {
                    const double gamma = dot_ew / n2_w;
                    double vp2 = fma(-(gamma * gamma), n2_w, n2_e);
                    if (vp2 < 0.0) vp2 = 0.0;
                    f->gain[o] = (float)gamma;
                    f->vpc[o] = (float)fma(-gamma, dot_cw, dot_ce);
                    perp[o] = (float)(sqrt(vp2) / sqrt_lm1);
                }
            }
        }
        /* banks, me8q_fast.cpp:240-302 */
        const size_t cnt = (size_t)(x->list_begin[c + 1] - x->list_begin[c]);
        for (size_t b = 0; b * 32 < cnt; ++b) {
            const size_t bi = f->batch0[c] + b;
            const size_t lo = (size_t)x->list_begin[c] + b * 32;
            const size_t m = cnt - b * 32 < 32 ? cnt - b * 32 : 32;
            for (int rr = 0; rr < nr; ++rr) {
                float vals[32][3], vmin[3] = {0, 0, 0}, vmax[3] = {0, 0, 0};
                for (size_t i = 0; i < m; ++i) {
                    const size_t pos = lo + i, o = pos * (size_t)nr + (size_t)rr;
                    const float coef = x->coef[pos * (size_t)x->ncoded + (size_t)f->rslot[rr]];
                    const float h2 = x->h2[pos * (size_t)x->ncoded + (size_t)f->rslot[rr]];
                    vals[i][0] = fmaf(-(2.0F * coef), f->vpc[o], h2);
                    vals[i][1] = 2.0F * coef * f->gain[o];
                    vals[i][2] = perp[o] * 2.0F * fabsf(coef);
                    for (int q = 0; q < 3; ++q) {
                        if (i == 0 || vals[i][q] < vmin[q]) vmin[q] = vals[i][q];
                        if (i == 0 || vals[i][q] > vmax[q]) vmax[q] = vals[i][q];
                    }
                }
                float sc[3];
                for (int q = 0; q < 3; ++q) sc[q] = vmax[q] > vmin[q] ? (vmax[q] - vmin[q]) / 255.0F : 1.0F;
                uint8_t* bp = f->bank + (bi * (size_t)nr + (size_t)rr) * 96;
                for (size_t i = 0; i < m; ++i) {
                    int v0 = (int)((vals[i][0] - vmin[0]) / sc[0]);
                    int v1 = (int)lroundf((vals[i][1] - vmin[1]) / sc[1]);
                    int v2 = (int)ceilf((vals[i][2] - vmin[2]) / sc[2]);
                    bp[i] = (uint8_t)(v0 < 0 ? 0 : (v0 > 255 ? 255 : v0));
                    bp[32 + i] = (uint8_t)(v1 < 0 ? 0 : (v1 > 255 ? 255 : v1));
                    bp[64 + i] = (uint8_t)(v2 < 0 ? 0 : (v2 > 255 ? 255 : v2));
                }
                float* sp = f->scl + (bi * (size_t)nr + (size_t)rr) * 6;
                sp[0] = vmin[0];
                sp[1] = sc[0];
                sp[2] = vmin[1];
                sp[3] = sc[1];
                sp[4] = vmin[2];
                sp[5] = sc[2];
            }
        }
    }
    free(perp);
}

/* ScoreRunSplitGeneric, src/simd/me8q_score_generic.cpp:100-126: the exact
 * fp32 score of one coded run (rate 1: one chain over the run; rate >= 2: a
 * chain per block, blocks summed). The split code decodes to the stored
 * digits, which are read here directly. */
static float run_score(const orc_me8q_index* x, const orc_fast* f, size_t pos, int r, const float* q) {
    const int bits = f->rbits[r], nblk = f->rlen[r] / 8;
    const uint16_t* dg = x->digits + pos * x->pd + f->roff[r];
    const uint8_t* br = x->branch + pos * (x->pd / 8) + f->roff[r] / 8;
    float acc = 0.0F;
    for (int blk = 0; blk < nblk; ++blk) {
        const float* lv = x->levf[bits][br[blk] ? 1 : 0];
        if (bits == 1) {
            for (int i = 0; i < 8; ++i) acc = fmaf(q[blk * 8 + i], lv[dg[blk * 8 + i]], acc);
        } else {
            float b = 0.0F;
            for (int i = 0; i < 8; ++i) b = fmaf(q[blk * 8 + i], lv[dg[blk * 8 + i]], b);
            acc += b;
        }
    }
    return acc;
}

/* PushCandidate, src/index/me8q_search.cpp:121-134. */
static void push_cand(float* hd, uint32_t* hi, size_t* cnt, size_t k, float dist, uint32_t id) {
    if (*cnt >= k && !(dist < hd[*cnt - 1])) return;
    if (*cnt >= k) --*cnt;
    size_t at = 0;
    while (at < *cnt && hd[at] < dist) ++at;
    memmove(hd + at + 1, hd + at, (*cnt - at) * sizeof(float));
    memmove(hi + at + 1, hi + at, (*cnt - at) * sizeof(uint32_t));
    hd[at] = dist;
    hi[at] = id;
    ++*cnt;
}

/* One kept lane waiting for the cascade (a member of flush4's group). */
typedef struct {
    size_t pos;
    double pool, qadd, sc[64], tr[64];
} orc_pending;

typedef struct {
    float* hd;
    uint32_t* hi;
    size_t cnt, k;
    uint64_t cand, surv;
} orc_heap;

/* flush4, src/index/me8q_fast.cpp:830-960: the group's runs in the order of
 * their mean t^2 per block (largest first; ties keep run order), each run's
 * exact score replacing its coarse term, death once the remaining slack
 * cannot bring the row under the heap's k-th distance. */
static void flush_group(const orc_me8q_index* x, const orc_fast* f, const float* rq, double d2, float lambda,
                        orc_pending* grp, int bn, orc_heap* h) {
    const int nr = f->nrun;
    int order[64];
    double mean[64];
    for (int r = 0; r < nr; ++r) {
        order[r] = r;
        mean[r] = 0.0;
        for (int j = 0; j < bn; ++j) mean[r] = fma(grp[j].tr[r], grp[j].tr[r], mean[r]);
        mean[r] /= (double)(f->rlen[r] / 8 > 1 ? f->rlen[r] / 8 : 1);
    }
    if (nr > 1)
        for (int a = 1; a < nr; ++a)
            for (int z = a; z > 0 && mean[order[z]] > mean[order[z - 1]]; --z) {
                const int t = order[z];
                order[z] = order[z - 1];
                order[z - 1] = t;
            }
    double dist[4], rem[4];
    int died[4] = {0, 0, 0, 0};
    for (int j = 0; j < bn; ++j) {
        const size_t ps = grp[j].pos;
        rem[j] = grp[j].pool;
        if (nr == 1) {
            dist[j] = d2 + (double)x->h2[ps * (size_t)x->ncoded + (size_t)f->rslot[0]];
        } else {
            double dcc = d2;
            for (int r = 0; r < nr; ++r) {
                const double coef = x->coef[ps * (size_t)x->ncoded + (size_t)f->rslot[r]];
                const double h2 = x->h2[ps * (size_t)x->ncoded + (size_t)f->rslot[r]];
                const size_t o = ps * (size_t)nr + (size_t)r;
                dcc += fma(-(2.0 * coef), fma((double)f->gain[o], grp[j].sc[r], (double)f->vpc[o]), h2);
            }
            dist[j] = dcc;
        }
    }
    const double dk = h->cnt < h->k ? INFINITY : (double)h->hd[h->cnt - 1];
    for (int oi = 0; oi < nr; ++oi) {
        const int r = order[oi];
        for (int j = 0; j < bn; ++j) {
            if (died[j]) continue;
            const size_t ps = grp[j].pos;
            const double coef = x->coef[ps * (size_t)x->ncoded + (size_t)f->rslot[r]];
            const double s_ex = (double)run_score(x, f, ps, r, rq + f->roff[r]);
            if (nr == 1) {
                dist[j] = fma(-(2.0 * coef), s_ex, dist[j]);
            } else {
                const size_t o = ps * (size_t)nr + (size_t)r;
                dist[j] = fma(2.0 * coef, fma((double)f->gain[o], grp[j].sc[r], (double)f->vpc[o]) - s_ex, dist[j]);
            }
            rem[j] = fma(-grp[j].tr[r], grp[j].tr[r], rem[j]);
            if (fma(-(double)lambda, sqrt(rem[j] > 0.0 ? rem[j] : 0.0), dist[j]) - grp[j].qadd >= dk) died[j] = 1;
        }
    }
    for (int j = 0; j < bn; ++j) {
        if (died[j]) continue;
        ++h->surv;
        push_cand(h->hd, h->hi, &h->cnt, h->k, (float)dist[j], x->ids[grp[j].pos]);
    }
}

/* ScanPreRouted, src/index/me8q_fast.cpp:548-1090, for one routed query: the
 * query LUT (one 64-entry line per plane column, quantised to u8 as
 * QuantizeLut does, src/simd/fastscan_avx512.cpp:12-39), per probed list the
 * coarse accumulators (AccumulateCoarseHi, src/simd/scan_kernels_generic.cpp:
 * 13-35), the coarse filter of CoarsePruneAvx512
 * (src/simd/me8q_prune_avx512.cpp:9-92: fp32, on the first 16*floor(m/16)
 * lanes of a batch of m) with its scalar fp64 twin on the tail lanes
 * (me8q_fast.cpp:985-1040), and the 4-wide run cascade against the live
 * heap. */
static void fast_query(const orc_me8q_index* x, const orc_fast* f, const float* rq, const float* d2l,
                       const uint64_t* keys, size_t take, float lambda, orc_heap* h) {
    const int nr = f->nrun, cols = f->cols;
    float* lut_f = (float*)calloc((size_t)cols * 64 + 1, sizeof(float));
    uint8_t* lut = (uint8_t*)calloc((size_t)cols * 64 + 1, 1);
    double qn2[64], lmx[64], qerr[64], smax[64], sd2[64];
    float delta = 1.0F;
    int lut_ready = 0;
    orc_pending grp[4];
    for (size_t p = 0; p < take; ++p) {
        const size_t c = (uint32_t)keys[p];
        const double d2 = (double)d2l[c];
        const size_t pb = (size_t)x->list_begin[c], lc = (size_t)(x->list_begin[c + 1] - pb);
        if (nr == 0) {  /* every dimension dropped: rows enter at d2 (:735-755) */
            for (size_t i = 0; i < lc; ++i) push_cand(h->hd, h->hi, &h->cnt, h->k, (float)d2, x->ids[pb + i]);
            h->cand += lc;
            h->surv += lc;
            continue;
        }
        if (lc == 0) continue;
        if (!lut_ready) {  /* prepare_list (:625-733), once: the plan is global */
            for (int r = 0; r < nr; ++r) {
                const int bits = f->rbits[r];
                const float p0 = f->pbar[bits][0], p1 = f->pbar[bits][1];
                const float p70 = bits == 1 ? 0.0F : p0, p71 = bits == 1 ? 0.0F : p1;
                for (int blk = 0; blk < f->rlen[r] / 8; ++blk) {
                    const float* qb = rq + f->roff[r] + blk * 8;
                    float* gl = lut_f + (size_t)(f->blk0[r] + blk) * 64;
                    float* gh = gl + 32;
                    for (int v = 0; v < 16; ++v) {
                        float a = qb[4] * (((v >> 3) & 1) ? p1 : p0);
                        a = fmaf(qb[5], ((v >> 2) & 1) ? p1 : p0, a);
                        a = fmaf(qb[6], ((v >> 1) & 1) ? p1 : p0, a);
                        gl[v] = fmaf(qb[7], (v & 1) ? p71 : p70, a);
                        float b = qb[0] * (((v >> 3) & 1) ? p1 : p0);
                        b = fmaf(qb[1], ((v >> 2) & 1) ? p1 : p0, b);
                        b = fmaf(qb[2], ((v >> 1) & 1) ? p1 : p0, b);
                        gh[v] = fmaf(qb[3], (v & 1) ? p1 : p0, b);
                    }
                    for (int v = 0; v < 16; ++v) {
                        gl[16 + v] = gl[v];
                        gh[16 + v] = gh[v];
                    }
                }
            }
            const size_t len = (size_t)cols * 64;
            float lo = lut_f[0], hv = lut_f[0];
            for (size_t i = 0; i < len; ++i) {
                if (lut_f[i] < lo) lo = lut_f[i];
                if (hv < lut_f[i]) hv = lut_f[i];
            }
            delta = hv > lo ? (hv - lo) / 255.0F : 1.0F;
            for (size_t i = 0; i < len; ++i) {
                const int v = (int)((lut_f[i] - lo) / delta + 0.5F);
                lut[i] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
            }
            for (int r = 0; r < nr; ++r) {
                double a = 0.0;
                for (int t = 0; t < f->rlen[r]; ++t) a = fma((double)rq[f->roff[r] + t], (double)rq[f->roff[r] + t], a);
                qn2[r] = a;
                const int nblk = f->rlen[r] / 8;
                lmx[r] = (double)lo * (2.0 * (double)nblk);
                const float sq = (float)sqrt((double)(nblk > 1 ? nblk : 1));
                qerr[r] = (double)(2.0F * sq * delta); /* LutErrClt, src/index/e8q_internal.hpp:107-109 */
                const double top = fma(2.0 * (double)nblk * 255.0, (double)delta, lmx[r]);
                smax[r] = fabs(lmx[r]) > fabs(top) ? fabs(lmx[r]) : fabs(top);
            }
            lut_ready = 1;
        }
        for (int r = 0; r < nr; ++r) {
            const float* rc = x->cent_rot + c * x->pd + f->roff[r];
            double dot = 0.0;
            for (int t = 0; t < f->rlen[r]; ++t) dot = fma((double)rq[f->roff[r] + t], (double)rc[t], dot);
            const double d2r = fma(-2.0, dot, qn2[r] + f->rc_n2[c * (size_t)nr + (size_t)r]);
            sd2[r] = sqrt(d2r > 0.0 ? d2r : 0.0);
        }
        for (size_t b = 0; b * 32 < lc; ++b) {
            const size_t m = lc - b * 32 < 32 ? lc - b * 32 : 32;
            const size_t bi = f->batch0[c] + b;
            static __thread int32_t acc[64][32];
            static __thread float lsc[64][32], ltr[64][32];
            for (int r = 0; r < nr; ++r)
                for (size_t l = 0; l < m; ++l) {
                    int32_t a = 0;
                    const uint8_t* row = f->plane + (pb + b * 32 + l) * (size_t)cols;
                    for (int blk = 0; blk < f->rlen[r] / 8; ++blk) {
                        const int col = f->blk0[r] + blk;
                        const uint8_t hb = row[col];
                        a += lut[(size_t)col * 64 + (hb & 15)] + lut[(size_t)col * 64 + 32 + (hb >> 4)];
                    }
                    acc[r][l] = a;
                }
            const size_t covered = m >= 16 ? (m / 16) * 16 : 0;
            const float distk0 = h->cnt < h->k ? INFINITY : h->hd[h->cnt - 1];
            float ldc[32], lpool[32], lqa[32];
            int keep[32];
            for (size_t l = 0; l < m; ++l) keep[l] = 1;
            if (covered) {
                const float sdk = distk0 < INFINITY ? sqrtf(distk0 > 0.0F ? distk0 : 0.0F) : INFINITY;
                for (size_t l = 0; l < covered; ++l) {
                    float dc = (float)d2, pool = 0.0F, qa = 0.0F, wpad = 0.0F;
                    for (int r = 0; r < nr; ++r) {
                        const uint8_t* bp = f->bank + (bi * (size_t)nr + (size_t)r) * 96;
                        const float* sc = f->scl + (bi * (size_t)nr + (size_t)r) * 6;
                        const float rh = sdk < (float)sd2[r] ? sdk : (float)sd2[r];
                        const float wp = (float)(0.5 * (double)sc[3] * (smax[r] + qerr[r]));
                        const float s_c = fmaf((float)acc[r][l], delta, (float)lmx[r]);
                        const float base_q = fmaf((float)bp[l], sc[1], sc[0]);
                        const float weight_q = fmaf((float)bp[32 + l], sc[3], sc[2]);
                        const float perp_q = fmaf((float)bp[64 + l], sc[5], sc[4]);
                        dc = fmaf(-weight_q, s_c, dc);
                        dc = dc + base_q;
                        const float t = perp_q * rh;
                        lsc[r][l] = s_c;
                        ltr[r][l] = t;
                        pool = fmaf(t, t, pool);
                        qa = fmaf(fabsf(weight_q), (float)qerr[r], qa);
                        wpad = wpad + wp;
                    }
                    const float slack = fmaf(lambda, sqrtf(pool), qa + wpad);
                    ldc[l] = dc;
                    lpool[l] = pool;
                    lqa[l] = qa + wpad;
                    if (dc - slack >= distk0) {
                        keep[l] = 0;
                        ++h->cand;
                    }
                }
            }
            int bn = 0;
            for (size_t l = 0; l < m; ++l) {
                if (!keep[l]) continue;
                const double distk = h->cnt < h->k ? INFINITY : (double)h->hd[h->cnt - 1];
                ++h->cand;
                double dc_q = d2, pool2 = 0.0, qadd = 0.0;
                orc_pending* g = &grp[bn];
                if (l < covered) {
                    dc_q = (double)ldc[l];
                    pool2 = (double)lpool[l];
                    qadd = (double)lqa[l];
                    for (int r = 0; r < nr; ++r) {
                        g->sc[r] = (double)lsc[r][l];
                        g->tr[r] = (double)ltr[r][l];
                    }
                } else {
                    const double sk = distk < INFINITY ? sqrt(distk > 0.0 ? distk : 0.0) : INFINITY;
                    for (int r = 0; r < nr; ++r) {
                        const uint8_t* bp = f->bank + (bi * (size_t)nr + (size_t)r) * 96;
                        const float* sc = f->scl + (bi * (size_t)nr + (size_t)r) * 6;
                        const double s_cr = fma((double)delta, (double)acc[r][l], lmx[r]);
                        g->sc[r] = s_cr;
                        const double base_q = fma((double)bp[l], (double)sc[1], (double)sc[0]);
                        const double weight_q = fma((double)bp[32 + l], (double)sc[3], (double)sc[2]);
                        const double perp_q = fma((double)bp[64 + l], (double)sc[5], (double)sc[4]);
                        dc_q += fma(-weight_q, s_cr, base_q);
                        const double rh = sk < sd2[r] ? sk : sd2[r];
                        g->tr[r] = perp_q * rh;
                        pool2 = fma(g->tr[r], g->tr[r], pool2);
                        qadd = fma(fabs(weight_q), qerr[r], qadd);
                        qadd = fma(0.5 * (double)sc[3], smax[r] + qerr[r], qadd);
                    }
                }
                if (dc_q - fma((double)lambda, sqrt(pool2), qadd) >= distk) continue;
                g->pos = pb + b * 32 + l;
                g->pool = pool2;
                g->qadd = qadd;
                if (++bn == 4) {
                    flush_group(x, f, rq, d2, lambda, grp, bn, h);
                    bn = 0;
                }
            }
            if (bn > 0) flush_group(x, f, rq, d2, lambda, grp, bn, h);
        }
    }
    free(lut_f);
    free(lut);
}

/* Me8qIndex.search (SearchIVFFast / SearchIVFFastBatch, the reference's
 * only search, python_bindings/me8q_bindings.cpp:97-160): route as
 * SearchIVF, then the FastScan cascade with lambda = OrthoQuantile(alpha,
 * max(4k, 32)) (alpha = the build's prune_alpha, 1 when not positive). Per
 * query the scanned candidates and the survivors pushed to the heap. */
void orc_me8q_search_pruned(const orc_me8q_index* x, const float* queries, size_t nq, size_t k, size_t nprobe,
                            float alpha, uint32_t* out_ids, float* out_dists, uint64_t* cand, uint64_t* surv,
                            int threads) {
    orc_fast f;
    fast_build(x, &f);
    const size_t ke = 4 * k > 32 ? 4 * k : 32;
    const float lambda = orc_ortho_quantile((double)(alpha > 0.0F ? alpha : 1.0F), ke);
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        float* qpad = (float*)malloc(sizeof(float) * x->pd);
        float* rq = (float*)malloc(sizeof(float) * x->pd);
        uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * x->nlist);
        float* d2 = (float*)malloc(sizeof(float) * x->nlist);
        orc_heap h;
        h.hd = (float*)malloc(sizeof(float) * (k + 1));
        h.hi = (uint32_t*)malloc(sizeof(uint32_t) * (k + 1));
        h.k = k;
#pragma omp for schedule(dynamic, 1)
        for (long long qi = 0; qi < (long long)nq; ++qi) {
            prepare_query(x, queries + (size_t)qi * x->dim, qpad, rq);
            route_query(x, rq, d2, keys);
            h.cnt = 0;
            h.cand = h.surv = 0;
            fast_query(x, &f, rq, d2, keys, nprobe < x->nlist ? nprobe : x->nlist, lambda, &h);
            for (size_t j = 0; j < k; ++j) {
                out_ids[(size_t)qi * k + j] = j < h.cnt ? h.hi[j] : 0xFFFFFFFFu;
                if (out_dists) out_dists[(size_t)qi * k + j] = j < h.cnt ? h.hd[j] : INFINITY;
            }
            if (cand) cand[qi] = h.cand;
            if (surv) surv[qi] = h.surv;
        }
        free(qpad);
        free(rq);
        free(keys);
        free(d2);
        free(h.hd);
        free(h.hi);
    }
    fast_free(&f);
}
