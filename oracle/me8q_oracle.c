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
