/* CPU oracle for the E8Q IVF search path -- TEST INFRASTRUCTURE ONLY.
 *
 * Restatement of the reference algorithm (paths relative to the reference
 * project). Compiled with -ffp-contract=off: every multiply-add the
 * reference's GCC -O3 build fuses (GCC's C++ default fp-contract=fast with an
 * FMA-capable -march) is written as an explicit fma() here, the rest stay
 * separate multiply and add. Products of two floats in double are exact, so
 * for those the choice does not matter.
 */
#include "e8q_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* sqrt(5/4): include/e8qlib/quantization/e8q_codec.hpp:24 */
static const double kSigmaC = 1.1180339887498949;

/* Acklam's rational approximation of the inverse normal CDF (P. J. Acklam,
 * 2003, published coefficients), as used by src/quantization/e8q_codec.cpp:17-44. */
double orc_inv_normal_cdf(double p) {
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02,
                                -2.759285104469687e+02, 1.383577518672690e+02,
                                -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02,
                                -1.556989798598866e+02, 6.680131188771972e+01,
                                -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01,
                                -2.400758277161838e+00, -2.549732539343734e+00,
                                4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01,
                                2.445134137142996e+00, 3.754408661907416e+00};
    const double plow = 0.02425;
    /* Horner chains as fused multiply-adds: the reference's build contracts
     * each `x * q + c` step into one FMA. */
    if (p < plow) {
        const double q = sqrt(-2 * log(p > 1e-300 ? p : 1e-300));
        const double num = fma(fma(fma(fma(fma(c[0], q, c[1]), q, c[2]), q, c[3]), q, c[4]), q, c[5]);
        const double den = fma(fma(fma(fma(d[0], q, d[1]), q, d[2]), q, d[3]), q, 1.0);
        return num / den;
    }
    if (p <= 1 - plow) {
        const double q = p - 0.5;
        const double r = q * q;
        const double num = fma(fma(fma(fma(fma(a[0], r, a[1]), r, a[2]), r, a[3]), r, a[4]), r, a[5]) * q;
        const double den = fma(fma(fma(fma(fma(b[0], r, b[1]), r, b[2]), r, b[3]), r, b[4]), r, 1.0);
        return num / den;
    }
    {
        const double omp = 1 - p;
        const double q = sqrt(-2 * log(omp > 1e-300 ? omp : 1e-300));
        const double num = fma(fma(fma(fma(fma(c[0], q, c[1]), q, c[2]), q, c[3]), q, c[4]), q, c[5]);
        const double den = fma(fma(fma(fma(d[0], q, d[1]), q, d[2]), q, d[3]), q, 1.0);
        return -num / den;
    }
}

/* BranchLevels: src/quantization/e8q_codec.cpp:496-509. Digit d holds the
 * quantile of t = start + i with d = t mod q. */
int orc_branch_levels(int bits, int branch, double* out) {
    const int q = 1 << bits;
    const double eta = 0.25 + 0.5 * (double)branch;
    const int start = (int)ceil(-0.5 * (double)q - eta);
    for (int i = 0; i < q; ++i) {
        const long t = (long)(start + i);
        const int digit = (int)(((t % q) + q) % q);
        double p = 0.5 + ((double)t + eta) / (double)q;
        p = p > 1e-12 ? p : 1e-12;
        p = p < 1.0 - 1e-12 ? p : 1.0 - 1e-12;
        out[digit] = kSigmaC * orc_inv_normal_cdf(p);
    }
    return q;
}

/* FixedScale: the per-rate scale schedule constants of
 * src/quantization/e8q_codec.cpp:456-460 (a codec constant; codes depend on it). */
double orc_fixed_scale(int bits) {
    static const double sched[ORC_MAX_BITS + 1] = {
        0.0, 1.118034, 0.895, 0.825, 0.785, 0.755, 0.735, 0.735,
        0.735, 0.725, 0.715, 0.705, 0.710, 0.705};
    if (bits < 1) return sched[1];
    if (bits > ORC_MAX_BITS) return sched[ORC_MAX_BITS];
    return sched[bits];
}

/* BuildRefineTables: src/quantization/e8q_codec.cpp:933-946. */
int orc_refine_tables(int bits, int padded_dim, float* out) {
    const int q = 1 << bits;
    const int stride = q > 256 ? q : 256;
    const double rd = sqrt((double)padded_dim);
    double* lev = (double*)malloc(sizeof(double) * (size_t)q);
    memset(out, 0, sizeof(float) * 2 * (size_t)stride);
    for (int br = 0; br < 2; ++br) {
        orc_branch_levels(bits, br, lev);
        for (int d = 0; d < q; ++d) out[br * stride + d] = (float)(lev[d] / rd);
    }
    free(lev);
    return 2 * stride;
}

/* ScanClassMeans: src/quantization/e8q_codec.cpp:511-524. */
void orc_scan_class_means(int bits, double w_cls[2]) {
    const int q = 1 << bits;
    double* l0 = (double*)malloc(sizeof(double) * (size_t)q);
    double* l1 = (double*)malloc(sizeof(double) * (size_t)q);
    orc_branch_levels(bits, 0, l0);
    orc_branch_levels(bits, 1, l1);
    const int cvals = 1 << (bits - 1);
    for (int t2 = 0; t2 < 2; ++t2) {
        double s0 = 0.0, s1 = 0.0;
        for (int lo = 0; lo < cvals; ++lo) {
            s0 += l0[(t2 << (bits - 1)) | lo];
            s1 += l1[(t2 << (bits - 1)) | lo];
        }
        w_cls[t2] = 0.5 * (s0 / cvals + s1 / cvals);
    }
    free(l0);
    free(l1);
}

/* ------------------------------------------------------------------------
 * Sorted level tables with the bounded-bin insertion index.
 * src/quantization/e8q_codec.cpp:70-123 (bin index), :125-186 (per-parity
 * tables), :283-352 (merged four-class table), :190-231 / :354-385 (insertion
 * point = std::lower_bound, via bins when usable, else binary search).
 * ---------------------------------------------------------------------- */
typedef struct {
    double* buf;      /* pad x -inf | n levels | pad x +inf */
    uint16_t* dig;    /* same indexing as buf */
    int pad;          /* leading pad entries */
    size_t n;
    uint32_t* bin_lo; /* nbins+1 */
    double bin_lo_v, bin_scale;
    size_t nbins;
    int usable;
    int alternating;  /* merged table only */
} level_table;

static void build_bin_index(level_table* t, size_t max_bins) {
    const double* lev = t->buf + t->pad;
    const size_t n = t->n;
    t->usable = 0;
    t->bin_lo = NULL;
    if (n < 16) return;
    const double lo_v = lev[0], hi_v = lev[n - 1];
    if (!(hi_v > lo_v)) return;
    double min_gap = DBL_MAX;
    for (size_t i = 1; i < n; ++i) {
        const double g = lev[i] - lev[i - 1];
        if (g < min_gap) min_gap = g;
    }
    if (!(min_gap > 0.0)) return;
    const double range = hi_v - lo_v;
    size_t bins = 1;
    while ((double)bins * min_gap < range && bins < max_bins) bins *= 2;
    if ((double)bins * min_gap < range) return;
    t->nbins = bins;
    t->bin_lo_v = lo_v;
    t->bin_scale = (double)bins / range;
    t->bin_lo = (uint32_t*)malloc(sizeof(uint32_t) * (bins + 1));
    size_t j = 0;
    for (size_t b = 0; b <= bins; ++b) {
        const double edge = lo_v + (double)b / t->bin_scale;
        while (j < n && lev[j] < edge) ++j;
        t->bin_lo[b] = (uint32_t)j;
    }
    size_t max_span = 0;
    for (size_t b = 0; b < bins; ++b) {
        const size_t sp = (size_t)(t->bin_lo[b + 1] - t->bin_lo[b]);
        if (sp > max_span) max_span = sp;
    }
    t->usable = max_span <= 2;
}

static size_t insert_pos(const level_table* t, double v) {
    const double* lev = t->buf + t->pad;
    const size_t n = t->n;
    if (t->usable) {
        if (v <= t->bin_lo_v) return 0;
        if (v > lev[n - 1]) return n;
        size_t bin = (size_t)((v - t->bin_lo_v) * t->bin_scale);
        if (bin >= t->nbins) bin = t->nbins - 1;
        size_t pos = t->bin_lo[bin];
        pos += (lev[pos] < v) ? 1 : 0;
        pos += (lev[pos] < v) ? 1 : 0;
        return pos;
    }
    size_t pos = 0, step = 1;
    while (step * 2 <= n) step *= 2;
    for (; step != 0; step >>= 1) {
        const size_t next = pos + step;
        pos += (next <= n && lev[next - 1] < v) ? step : 0;
    }
    return pos;
}

typedef struct {
    double v;
    uint16_t dig;
    uint8_t branch;
    uint32_t order; /* original index: makes qsort stable */
} merged_entry;

static int cmp_merged(const void* a, const void* b) {
    const merged_entry* x = (const merged_entry*)a;
    const merged_entry* y = (const merged_entry*)b;
    if (x->v < y->v) return -1;
    if (y->v < x->v) return 1;
    return x->order < y->order ? -1 : (x->order > y->order ? 1 : 0);
}

static level_table g_merged[ORC_MAX_BITS + 1];
static level_table g_parity[ORC_MAX_BITS + 1][2][2];
static int g_merged_ready[ORC_MAX_BITS + 1];
static int g_parity_ready[ORC_MAX_BITS + 1][2][2];
static double* g_levels[ORC_MAX_BITS + 1][2];

static const double* levels_of(int bits, int br) {
    if (g_levels[bits][br] == NULL) {
        double* l = (double*)malloc(sizeof(double) * ((size_t)1 << bits));
        orc_branch_levels(bits, br, l);
        g_levels[bits][br] = l;
    }
    return g_levels[bits][br];
}

/* GetMergedTable: src/quantization/e8q_codec.cpp:297-352. */
static const level_table* merged_table(int bits) {
    if (g_merged_ready[bits]) return &g_merged[bits];
    const size_t q = (size_t)1 << bits;
    const size_t n = 2 * q;
    const double* l0 = levels_of(bits, 0);
    const double* l1 = levels_of(bits, 1);
    merged_entry* raw = (merged_entry*)malloc(sizeof(merged_entry) * n);
    for (size_t d = 0; d < q; ++d) {
        raw[2 * d] = (merged_entry){l0[d], (uint16_t)d, 0, (uint32_t)(2 * d)};
        raw[2 * d + 1] = (merged_entry){l1[d], (uint16_t)d, 1, (uint32_t)(2 * d + 1)};
    }
    qsort(raw, n, sizeof(merged_entry), cmp_merged);
    int alt = 1;
    for (size_t i = 0; i < n; ++i) {
        if (i > 0 && !(raw[i].v > raw[i - 1].v)) { alt = 0; break; }
        if (raw[i].branch != (uint8_t)(i & 1u) || (raw[i].dig & 1u) != ((i >> 1) & 1u)) {
            alt = 0;
            break;
        }
    }
    level_table* t = &g_merged[bits];
    t->pad = 4;
    t->n = n;
    t->alternating = alt;
    t->buf = (double*)malloc(sizeof(double) * (n + 8));
    t->dig = (uint16_t*)calloc(n + 8, sizeof(uint16_t));
    for (int i = 0; i < 4; ++i) {
        t->buf[i] = -INFINITY;
        t->buf[n + 4 + i] = INFINITY;
    }
    for (size_t i = 0; i < n; ++i) {
        t->buf[4 + i] = raw[i].v;
        t->dig[4 + i] = raw[i].dig;
    }
    t->usable = 0;
    t->bin_lo = NULL;
    if (alt) build_bin_index(t, 32768);
    free(raw);
    g_merged_ready[bits] = 1;
    return t;
}

/* GetParityTable: src/quantization/e8q_codec.cpp:142-186. */
static const level_table* parity_table(int bits, int branch, int odd) {
    if (g_parity_ready[bits][branch][odd]) return &g_parity[bits][branch][odd];
    const int q = 1 << bits;
    const double* levels = levels_of(bits, branch);
    level_table* t = &g_parity[bits][branch][odd];
    const size_t n = (size_t)(q / 2);
    t->pad = 0;
    t->n = n;
    t->buf = (double*)malloc(sizeof(double) * (n + 2));
    t->dig = (uint16_t*)calloc(n + 2, sizeof(uint16_t));
    size_t m = 0;
    for (int d = odd ? 1 : 0; d < q; d += 2) {
        t->buf[m] = levels[d];
        t->dig[m] = (uint16_t)d;
        ++m;
    }
    for (size_t i = 1; i < n; ++i) { /* insertion sort by (level, digit) */
        const double lv = t->buf[i];
        const uint16_t dg = t->dig[i];
        size_t j = i;
        while (j > 0 && (t->buf[j - 1] > lv || (t->buf[j - 1] == lv && t->dig[j - 1] > dg))) {
            t->buf[j] = t->buf[j - 1];
            t->dig[j] = t->dig[j - 1];
            --j;
        }
        t->buf[j] = lv;
        t->dig[j] = dg;
    }
    build_bin_index(t, 16384);
    t->buf[n] = INFINITY;
    t->buf[n + 1] = INFINITY;
    g_parity_ready[bits][branch][odd] = 1;
    return t;
}

int orc_merged_alternating(int bits) { return merged_table(bits)->alternating; }

/* Pre-build every table once (the encoder then only reads them, so OpenMP
 * threads can share them). */
static void warm_tables(int bits) {
    const level_table* mt = merged_table(bits);
    if (!mt->alternating) {
        for (int br = 0; br < 2; ++br)
            for (int od = 0; od < 2; ++od) parity_table(bits, br, od);
    }
}

void orc_warm_tables(int bits) { warm_tables(bits); }

/* NearestInTable: src/quantization/e8q_codec.cpp:233-256. */
static void nearest_in_table(double v, const level_table* t, uint16_t* digit, double* cost) {
    const double* lev = t->buf;
    const size_t n = t->n;
    const size_t pos = insert_pos(t, v);
    size_t best = pos < n ? pos : n - 1;
    if (pos > 0) {
        const double dc = fabs(v - lev[pos - 1]);
        const double db = fabs(v - lev[best]);
        const uint16_t dig_c = t->dig[pos - 1];
        const uint16_t dig_b = t->dig[best];
        const int take_below = (dc < db) | ((dc == db) & (dig_c < dig_b));
        best = take_below ? pos - 1 : best;
    }
    *digit = t->dig[best];
    const double dv = v - lev[best];
    *cost = dv * dv;
}

/* NearestMerged: src/quantization/e8q_codec.cpp:392-414. Class r = 2*parity +
 * branch sits at merged positions i with (i & 3) == r. */
static void nearest_merged(double v, const level_table* t, uint16_t dig[4], double cost[4]) {
    const double* lev = t->buf + t->pad;
    const uint16_t* dg = t->dig + t->pad;
    const long p = (long)insert_pos(t, v);
    const long p4 = p & 3;
    for (long r = 0; r < 4; ++r) {
        const long i_b = p - 1 - ((p4 + 3 - r) & 3);
        const long i_a = p + ((r + 4 - p4) & 3);
        const uint16_t d_b = dg[i_b];
        const uint16_t d_a = dg[i_a];
        const double dv_b = v - lev[i_b];
        const double dv_a = lev[i_a] - v;
        const double c_b = dv_b * dv_b;
        const double c_a = dv_a * dv_a;
        const int take_b = (c_b < c_a) | ((c_b == c_a) & (d_b < d_a));
        dig[r] = take_b ? d_b : d_a;
        cost[r] = take_b ? c_b : c_a;
    }
}

typedef struct {
    uint16_t digits[8];
    double cost;
} block_code;

/* AssembleBlock: per-coordinate parity choice + single-flip parity repair,
 * src/quantization/e8q_codec.cpp:549-599. */
static block_code assemble_block(const uint16_t dig_e[8], const double cost_e[8],
                                 const uint16_t dig_o[8], const double cost_o[8]) {
    block_code out;
    out.cost = 0.0;
    int parity = 0;
    for (int i = 0; i < 8; ++i) {
        const int use_odd = cost_o[i] < cost_e[i];
        out.digits[i] = use_odd ? dig_o[i] : dig_e[i];
        out.cost += use_odd ? cost_o[i] : cost_e[i];
        parity ^= use_odd;
    }
    if (parity != 0) {
        int sel = 0;
        double best_extra = DBL_MAX;
        for (int i = 0; i < 8; ++i) {
            const int was_odd = out.digits[i] == dig_o[i];
            const double extra = was_odd ? cost_e[i] - cost_o[i] : cost_o[i] - cost_e[i];
            if (extra < best_extra) {
                best_extra = extra;
                sel = i;
            }
        }
        const int was_odd = out.digits[sel] == dig_o[sel];
        out.digits[sel] = was_odd ? dig_e[sel] : dig_o[sel];
        out.cost += (best_extra < 0.0) ? 0.0 : best_extra;
    }
    return out;
}

/* EncodeVectorAtScaleInto: src/quantization/e8q_codec.cpp:671-726. */
void orc_encode(const float* unit, size_t n, int padded_dim, int bits, double s,
                uint16_t* digits, uint8_t* branch) {
    warm_tables(bits);
    const int blocks = padded_dim / 8;
    const double rd = sqrt((double)padded_dim);
    const double srd = s * rd;
    const level_table* mt = merged_table(bits);
    for (size_t r = 0; r < n; ++r) {
        const float* u = unit + r * (size_t)padded_dim;
        for (int blk = 0; blk < blocks; ++blk) {
            double v[8];
            for (int i = 0; i < 8; ++i) v[i] = (double)u[blk * 8 + i] * srd;
            block_code e0, e1;
            if (mt->alternating) {
                uint16_t de0[8], do0[8], de1[8], do1[8];
                double ce0[8], co0[8], ce1[8], co1[8];
                for (int i = 0; i < 8; ++i) {
                    uint16_t dg[4];
                    double cs[4];
                    nearest_merged(v[i], mt, dg, cs);
                    de0[i] = dg[0]; ce0[i] = cs[0];
                    de1[i] = dg[1]; ce1[i] = cs[1];
                    do0[i] = dg[2]; co0[i] = cs[2];
                    do1[i] = dg[3]; co1[i] = cs[3];
                }
                e0 = assemble_block(de0, ce0, do0, co0);
                e1 = assemble_block(de1, ce1, do1, co1);
            } else {
                block_code e[2];
                for (int br = 0; br < 2; ++br) {
                    uint16_t de[8], dodd[8];
                    double ce[8], co[8];
                    const level_table* te = parity_table(bits, br, 0);
                    const level_table* to = parity_table(bits, br, 1);
                    for (int i = 0; i < 8; ++i) {
                        nearest_in_table(v[i], te, &de[i], &ce[i]);
                        nearest_in_table(v[i], to, &dodd[i], &co[i]);
                    }
                    e[br] = assemble_block(de, ce, dodd, co);
                }
                e0 = e[0];
                e1 = e[1];
            }
            const int take1 = e1.cost < e0.cost;
            uint16_t* dst = digits + ((r * (size_t)blocks) + (size_t)blk) * 8;
            memcpy(dst, take1 ? e1.digits : e0.digits, sizeof(uint16_t) * 8);
            branch[r * (size_t)blocks + (size_t)blk] = (uint8_t)take1;
        }
    }
}

/* PackCoarseRow: src/index/e8q_scan.cpp:15-27. */
uint8_t orc_pack_coarse(const uint16_t digits[8], int branch, int bits) {
    uint8_t byte = 0;
    for (int i = 0; i < 8; ++i) {
        const int top = (bits == 1 && i == 7) ? (branch & 1) : ((digits[i] >> (bits - 1)) & 1);
        if (top) byte |= (uint8_t)(1u << (7 - i));
    }
    return byte;
}

/* PackRefineBlock (b >= 2): src/quantization/e8q_codec.cpp:827-838. Low c = b-1
 * bits of digits 0..6 little-endian, digit 7's bit 0 replaced by the branch. */
void orc_pack_refine(const uint16_t digits[8], int branch, int bits, uint8_t* out) {
    if (bits < 2) return;
    const int c = bits - 1;
    uint8_t acc[16] = {0};
    for (int i = 0; i < 8; ++i) {
        uint32_t f = (uint32_t)digits[i] & ((1u << c) - 1u);
        if (i == 7) f = (f & ~1u) | (uint32_t)(branch & 1);
        for (int bit = 0; bit < c; ++bit) {
            if ((f >> bit) & 1u) {
                const int pos = c * i + bit;
                acc[pos >> 3] |= (uint8_t)(1u << (pos & 7));
            }
        }
    }
    memcpy(out, acc, (size_t)c);
}

/* DecodeSplitBlockLane: src/index/e8q_scan.cpp:34-87 (b >= 2) and the b == 1
 * sign-byte form of src/quantization/e8q_codec.cpp:856-870. */
void orc_decode_split(int bits, uint8_t rowa, const uint8_t* refine, uint16_t digits[8],
                      int* branch) {
    if (bits == 1) {
        int par = 0;
        for (int i = 0; i < 7; ++i) {
            digits[i] = (uint16_t)((rowa >> (7 - i)) & 1u);
            par ^= digits[i] & 1;
        }
        digits[7] = (uint16_t)par;
        *branch = rowa & 1;
        return;
    }
    const int c = bits - 1;
    int par = 0;
    uint32_t f[8];
    for (int i = 0; i < 8; ++i) {
        uint32_t v = 0;
        for (int bit = 0; bit < c; ++bit) {
            const int pos = c * i + bit;
            v |= (uint32_t)((refine[pos >> 3] >> (pos & 7)) & 1u) << bit;
        }
        f[i] = v;
    }
    for (int i = 0; i < 7; ++i) {
        digits[i] = (uint16_t)(f[i] | ((uint32_t)((rowa >> (7 - i)) & 1u) << c));
        par ^= (int)(f[i] & 1u);
    }
    digits[7] = (uint16_t)(((f[7] >> 1) << 1) | (uint32_t)par | ((uint32_t)(rowa & 1u) << c));
    *branch = (int)(f[7] & 1u);
}

/* ------------------------------------------------------------------------
 * FHT-Kac-4 rotator: src/utils/rotator.cpp:13-80, primitives
 * src/simd/kernels_generic.cpp:49-77.
 * ---------------------------------------------------------------------- */

/* MT19937-64 (Matsumoto & Nishimura; the parameters std::mt19937_64 fixes). */
typedef struct {
    uint64_t mt[312];
    int idx;
} mt64;

static void mt64_seed(mt64* g, uint64_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->idx = 312;
}

static uint64_t mt64_next(mt64* g) {
    if (g->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            const uint64_t x = (g->mt[i] & 0xFFFFFFFF80000000ULL) |
                               (g->mt[(i + 1) % 312] & 0x7FFFFFFFULL);
            uint64_t xa = x >> 1;
            if (x & 1ULL) xa ^= 0xB5026F5AA96619E9ULL;
            g->mt[i] = g->mt[(i + 156) % 312] ^ xa;
        }
        g->idx = 0;
    }
    uint64_t y = g->mt[g->idx++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= y >> 43;
    return y;
}

size_t orc_padded_dim(size_t dim) { return (dim + 63) / 64 * 64; }
size_t orc_sign_bytes(size_t dim) { return 4 * orc_padded_dim(dim) / 8; }

/* Sign bytes: one uniform draw in [0, 255] per byte from mt19937_64(seed).
 * For a 256-wide range of a full 64-bit engine the standard library's
 * multiply-shift reduction (Lemire 2019) returns the top 8 bits of the draw,
 * with no rejection (256 divides 2^64). */
void orc_rotator_signs(size_t dim, uint64_t seed, uint8_t* out) {
    mt64 g;
    mt64_seed(&g, seed);
    const size_t nb = orc_sign_bytes(dim);
    for (size_t i = 0; i < nb; ++i) out[i] = (uint8_t)(mt64_next(&g) >> 56);
}

static void fht(float* buf, size_t len) {
    for (size_t h = 1; h < len; h <<= 1)
        for (size_t i = 0; i < len; i += h << 1)
            for (size_t j = 0; j < h; ++j) {
                const float x = buf[i + j];
                const float y = buf[i + j + h];
                buf[i + j] = x + y;
                buf[i + j + h] = x - y;
            }
}

static size_t trunc_dim(size_t dim) {
    size_t bl = 0;
    while (((size_t)1 << (bl + 1)) <= dim) ++bl;
    return (size_t)1 << bl;
}

void orc_rotate(size_t dim, const uint8_t* signs, const float* src, float* dst) {
    const size_t pd = orc_padded_dim(dim);
    const size_t td = trunc_dim(dim);
    const float fac = 1.0F / sqrtf((float)td);
    memcpy(dst, src, sizeof(float) * dim);
    memset(dst + dim, 0, sizeof(float) * (pd - dim));
    const size_t per_round = pd / 8;
    for (int r = 0; r < 4; ++r) {
        const uint8_t* sg = signs + (size_t)r * per_round;
        for (size_t i = 0; i < pd; ++i)
            if ((sg[i / 8] >> (i % 8)) & 1) dst[i] = -dst[i];
        float* win = dst + ((td == pd || r % 2 == 0) ? 0 : pd - td);
        fht(win, td);
        for (size_t i = 0; i < td; ++i) win[i] *= fac;
        if (td != pd) {
            const size_t half = pd / 2;
            for (size_t i = 0; i < half; ++i) {
                const float x = dst[i], y = dst[i + half];
                dst[i] = x + y;
                dst[i + half] = x - y;
            }
        }
    }
    if (td != pd)
        for (size_t i = 0; i < pd; ++i) dst[i] *= 0.25F;
}

/* ------------------------------------------------------------------------
 * Index build, restating src/index/e8q_build.cpp:87-418 for the state the
 * plain search reads (codes, g1, h3, ids, rotated centroids, norms, mean).
 * ---------------------------------------------------------------------- */
orc_e8q_index* orc_e8q_build(const float* base, const float* centroids,
                             const uint32_t* cluster_ids, size_t n, size_t dim,
                             size_t nlist, int bits, uint64_t seed, int threads) {
    if (bits < 1 || bits > ORC_MAX_BITS || n == 0 || nlist == 0 || dim == 0) return NULL;
    for (size_t i = 0; i < n; ++i)
        if (cluster_ids[i] >= nlist) return NULL;
    warm_tables(bits);
    orc_e8q_index* x = (orc_e8q_index*)calloc(1, sizeof(orc_e8q_index));
    const size_t pd = orc_padded_dim(dim);
    const int B = (int)(pd / 8);
    x->n = n; x->dim = dim; x->padded_dim = pd; x->nlist = nlist; x->bits = bits; x->blocks = B;
    x->signs = (uint8_t*)malloc(orc_sign_bytes(dim));
    orc_rotator_signs(dim, seed, x->signs);
    x->tab_stride = (1 << bits) > 256 ? (1 << bits) : 256;
    x->tab = (float*)malloc(sizeof(float) * 2 * (size_t)x->tab_stride);
    orc_refine_tables(bits, (int)pd, x->tab);

    /* posting lists in file order: :120-133, :225-231 */
    x->list_begin = (uint64_t*)calloc(nlist + 1, sizeof(uint64_t));
    for (size_t i = 0; i < n; ++i) x->list_begin[cluster_ids[i] + 1]++;
    for (size_t c = 0; c < nlist; ++c) x->list_begin[c + 1] += x->list_begin[c];
    uint64_t* cursor = (uint64_t*)malloc(sizeof(uint64_t) * nlist);
    memcpy(cursor, x->list_begin, sizeof(uint64_t) * nlist);
    size_t* slot = (size_t*)malloc(sizeof(size_t) * n);
    x->ids = (uint32_t*)malloc(sizeof(uint32_t) * n);
    for (size_t i = 0; i < n; ++i) {
        slot[i] = cursor[cluster_ids[i]]++;
        x->ids[slot[i]] = (uint32_t)i;
    }
    free(cursor);

    /* mean in fp64, file order, then rotated: :190-204 */
    double* mu = (double*)calloc(dim, sizeof(double));
    for (size_t i = 0; i < n; ++i)
        for (size_t d = 0; d < dim; ++d) mu[d] += (double)base[i * dim + d];
    float* mu_f = (float*)malloc(sizeof(float) * dim);
    for (size_t d = 0; d < dim; ++d) mu_f[d] = (float)(mu[d] / (double)n);
    x->mean_rot = (float*)malloc(sizeof(float) * pd);
    orc_rotate(dim, x->signs, mu_f, x->mean_rot);
    free(mu);
    free(mu_f);

    /* rotated, centred centroids + fp64 norms: :249-272 */
    x->centroid_rot = (float*)malloc(sizeof(float) * nlist * pd);
    x->cn2 = (float*)malloc(sizeof(float) * nlist);
    for (size_t c = 0; c < nlist; ++c) {
        float* rc = x->centroid_rot + c * pd;
        orc_rotate(dim, x->signs, centroids + c * dim, rc);
        double s2 = 0.0;
        for (size_t d = 0; d < pd; ++d) {
            rc[d] -= x->mean_rot[d];
            s2 = fma((double)rc[d], (double)rc[d], s2);
        }
        x->cn2[c] = (float)s2;
    }

    x->digits = (uint16_t*)calloc(n * (size_t)B * 8, sizeof(uint16_t));
    x->branch = (uint8_t*)calloc(n * (size_t)B, 1);
    x->g1 = (float*)calloc(n, sizeof(float));
    x->h3 = (float*)calloc(n, sizeof(float));
    x->ortho = (float*)calloc(n * 3, sizeof(float));
    double w_cls[2];
    orc_scan_class_means(bits, w_cls);
    const double sqrt_dm1 = sqrt((double)(dim > 1 ? dim - 1 : 1));
    const double s_vec = orc_fixed_scale(bits);
    const double inv_level_scale = 1.0 / sqrt((double)pd);
    const double* lev[2] = {levels_of(bits, 0), levels_of(bits, 1)};

    /* encode + fit per row: :306-418 */
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        float* rot_x = (float*)malloc(sizeof(float) * pd);
        float* unit = (float*)malloc(sizeof(float) * pd);
#pragma omp for schedule(dynamic, 256)
        for (long long ri = 0; ri < (long long)n; ++ri) {
            const size_t row = (size_t)ri;
            const size_t pos = slot[row];
            const float* rc = x->centroid_rot + (size_t)cluster_ids[row] * pd;
            orc_rotate(dim, x->signs, base + row * dim, rot_x);
            for (size_t d = 0; d < pd; ++d) rot_x[d] -= x->mean_rot[d];
            double rn2 = 0.0;
            for (size_t d = 0; d < pd; ++d) {
                const double rv = (double)rot_x[d] - (double)rc[d];
                rn2 = fma(rv, rv, rn2);
            }
            const double rn = sqrt(rn2);
            if (rn < 1e-20) continue; /* codes, g1, h3 stay zero: :317-322 */
            const double inv_rn = 1.0 / rn;
            for (size_t d = 0; d < pd; ++d)
                unit[d] = (float)(((double)rot_x[d] - (double)rc[d]) * inv_rn);
            uint16_t* dg = x->digits + pos * (size_t)B * 8;
            uint8_t* br = x->branch + pos * (size_t)B;
            orc_encode(unit, 1, (int)pd, bits, s_vec, dg, br);
            /* scan-basis projections: w is the branch-averaged class mean of
             * each digit's top bit, none for dim 7 at b = 1 (:338-377) */
            double dot_ue = 0.0, n2_e = 0.0, dot_ce = 0.0;
            double dot_ew = 0.0, dot_uw = 0.0, n2_w = 0.0, dot_cw = 0.0;
            for (int blk = 0; blk < B; ++blk) {
                for (int k = 0; k < 8; ++k) {
                    const int digit = dg[blk * 8 + k];
                    const double ve = lev[br[blk]][digit] * inv_level_scale;
                    const double wc = (bits == 1 && k == 7) ? 0.0 : w_cls[digit >> (bits - 1)];
                    const size_t idx = (size_t)blk * 8 + (size_t)k;
                    dot_ue = fma((double)unit[idx], ve, dot_ue);
                    dot_ce = fma((double)rc[idx], ve, dot_ce);
                    n2_e = fma(ve, ve, n2_e);
                    dot_ew = fma(ve, wc, dot_ew);
                    dot_uw = fma((double)unit[idx], wc, dot_uw);
                    n2_w = fma(wc, wc, n2_w);
                    dot_cw = fma((double)rc[idx], wc, dot_cw);
                }
            }
            double g1 = 0.0, h3 = 0.0;
            if (n2_e > 1e-30 && dot_ue > 1e-12) {
                g1 = rn / dot_ue;
                h3 = fma(2.0 * g1, dot_ce, rn2);
            }
            x->g1[pos] = (float)g1;
            x->h3[pos] = (float)h3;
            /* zero-parallel-residual bank inputs (:405-445) with the fused
             * multiply-adds the reference's GCC build forms: rx2 as
             * fnma(c1, <e,w>, fma(a1, |e|^2, b1*|w|^2)), vp2 and base as one
             * fma each */
            {
                const double g1v = (double)x->g1[pos];
                const double n2_w_safe = n2_w < 1e-30 ? 1e-30 : n2_w;
                const double uw_eps = 1e-12 * sqrt(n2_w_safe);
                double w_use, perp_use;
                if (fabs(dot_uw) > uw_eps) {
                    const double wx = 2.0 * rn / dot_uw;
                    const double a1 = 4.0 * g1v * g1v, b1 = wx * wx, c1 = 4.0 * g1v * wx;
                    const double rx2 = fma(-c1, dot_ew, fma(a1, n2_e, b1 * n2_w));
                    w_use = wx;
                    perp_use = sqrt(0.0 < rx2 ? rx2 : 0.0) / sqrt_dm1;
                } else {
                    const double gamma = dot_ew / n2_w_safe;
                    const double t = fma(-(gamma * gamma), n2_w, n2_e);
                    const double vp2 = t < 0.0 ? 0.0 : t;
                    w_use = 2.0 * g1v * gamma;
                    perp_use = 2.0 * g1v * sqrt(vp2) / sqrt_dm1;
                }
                x->ortho[pos * 3 + 0] = (float)fma(w_use, dot_cw, rn2);
                x->ortho[pos * 3 + 1] = (float)w_use;
                x->ortho[pos * 3 + 2] = (float)perp_use;
            }
        }
        free(rot_x);
        free(unit);
    }
    free(slot);
    return x;
}

void orc_e8q_free(orc_e8q_index* x) {
    if (!x) return;
    free(x->signs); free(x->mean_rot); free(x->centroid_rot); free(x->cn2);
    free(x->list_begin); free(x->ids); free(x->digits); free(x->branch);
    free(x->g1); free(x->h3); free(x->tab); free(x->ortho);
    free(x);
}

/* rotate + subtract rot(mu): src/index/e8q_search.cpp:242-246 */
void orc_e8q_prepare_query(const orc_e8q_index* x, const float* q, float* rot_q) {
    orc_rotate(x->dim, x->signs, q, rot_q);
    for (size_t d = 0; d < x->padded_dim; ++d) rot_q[d] -= x->mean_rot[d];
}

/* ExactScore: src/index/e8q_search.cpp:87-127 (fp64 accumulation of
 * q[i] * table[br][digit]; a float*float product is exact in double). */
float orc_e8q_exact_score(const orc_e8q_index* x, size_t pos, const float* rot_q) {
    const uint16_t* dg = x->digits + pos * (size_t)x->blocks * 8;
    const uint8_t* br = x->branch + pos * (size_t)x->blocks;
    double acc = 0.0;
    for (int blk = 0; blk < x->blocks; ++blk) {
        const float* tab = x->tab + (size_t)br[blk] * (size_t)x->tab_stride;
        for (int d = 0; d < 8; ++d)
            acc += (double)rot_q[blk * 8 + d] * (double)tab[dg[blk * 8 + d]];
    }
    return (float)acc;
}

static size_t list_of(const orc_e8q_index* x, size_t pos) {
    size_t lo = 0, hi = x->nlist;
    while (hi - lo > 1) {
        const size_t mid = (lo + hi) / 2;
        if (x->list_begin[mid] <= pos) lo = mid; else hi = mid;
    }
    return lo;
}

/* Estimate: src/index/e8q_oracle.cpp:58-101 (fp32 qn2/dot chains, which the
 * reference build fuses into FMAs). */
float orc_e8q_estimate(const orc_e8q_index* x, const float* q, uint32_t id) {
    size_t pos = (size_t)-1;
    for (size_t i = 0; i < x->n; ++i)
        if (x->ids[i] == id) { pos = i; break; }
    if (pos == (size_t)-1) return NAN;
    const size_t c = list_of(x, pos);
    float* rq = (float*)malloc(sizeof(float) * x->padded_dim);
    orc_e8q_prepare_query(x, q, rq);
    float qn2 = 0.0F, dot = 0.0F;
    const float* cc = x->centroid_rot + c * x->padded_dim;
    for (size_t d = 0; d < x->padded_dim; ++d) {
        qn2 = fmaf(rq[d], rq[d], qn2);
        dot = fmaf(rq[d], cc[d], dot);
    }
    float d2 = fmaf(-2.0F, dot, qn2 + x->cn2[c]);
    if (d2 < 0.0F) d2 = 0.0F;
    const float s = orc_e8q_exact_score(x, pos, rq);
    free(rq);
    return fmaf(-(2.0F * x->g1[pos]), s, d2 + x->h3[pos]);
}

/* RouteL2 with the scalar GEMV: src/index/ivf_route.cpp:9-27,
 * src/simd/kernels_generic.cpp:5-33, key packing src/simd/kernels.hpp:13-21. */
static void route_keys(const orc_e8q_index* x, const float* rq, uint64_t* keys, float* d2) {
    double s = 0.0;
    for (size_t d = 0; d < x->padded_dim; ++d) s += (double)rq[d] * (double)rq[d];
    const float qn2 = (float)s;
    for (size_t c = 0; c < x->nlist; ++c) {
        const float* cc = x->centroid_rot + c * x->padded_dim;
        double dot = 0.0;
        for (size_t d = 0; d < x->padded_dim; ++d) dot += (double)rq[d] * (double)cc[d];
        float v = fmaf(-2.0F, (float)dot, qn2 + x->cn2[c]);
        if (v < 0.0F) v = 0.0F;
        d2[c] = v;
        uint32_t bitsv;
        memcpy(&bitsv, &v, 4);
        keys[c] = ((uint64_t)bitsv << 32) | (uint64_t)c;
    }
}

static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

void orc_e8q_route(const orc_e8q_index* x, const float* rq, size_t nprobe,
                   uint32_t* probe_ids, float* probe_d2) {
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * x->nlist);
    float* d2 = (float*)malloc(sizeof(float) * x->nlist);
    route_keys(x, rq, keys, d2);
    qsort(keys, x->nlist, sizeof(uint64_t), cmp_u64);
    const size_t take = nprobe < x->nlist ? nprobe : x->nlist;
    for (size_t p = 0; p < take; ++p) {
        probe_ids[p] = (uint32_t)keys[p];
        if (probe_d2) probe_d2[p] = d2[(uint32_t)keys[p]];
    }
    free(keys);
    free(d2);
}

/* Better(): src/index/e8q_internal.hpp:47-49 */
static int better(float d1, uint32_t i1, float d2, uint32_t i2) {
    return d1 < d2 || (d1 == d2 && i1 < i2);
}

/* Size-k heap + sorted extraction: src/index/e8q_search.cpp:135-180, 295-318.
 * Plain mode: every candidate of every probed list is scored exactly
 * (the disable_prune mask, src/simd/e8q_search_avx512.cpp:668-669). */
void orc_e8q_search(const orc_e8q_index* x, const float* queries, size_t nq, size_t k,
                    size_t nprobe, uint32_t* out_ids, float* out_dists, int threads) {
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        float* rq = (float*)malloc(sizeof(float) * x->padded_dim);
        uint32_t* probes = (uint32_t*)malloc(sizeof(uint32_t) * x->nlist);
        float* pd2 = (float*)malloc(sizeof(float) * x->nlist);
        float* hd = (float*)malloc(sizeof(float) * (k + 1));
        uint32_t* hi = (uint32_t*)malloc(sizeof(uint32_t) * (k + 1));
#pragma omp for schedule(dynamic, 1)
        for (long long qi = 0; qi < (long long)nq; ++qi) {
            orc_e8q_prepare_query(x, queries + (size_t)qi * x->dim, rq);
            const size_t take = nprobe < x->nlist ? nprobe : x->nlist;
            orc_e8q_route(x, rq, take, probes, pd2);
            size_t cnt = 0;
            for (size_t p = 0; p < take; ++p) {
                const size_t c = probes[p];
                const float d2 = pd2[p];
                for (uint64_t pos = x->list_begin[c]; pos < x->list_begin[c + 1]; ++pos) {
                    const float s = orc_e8q_exact_score(x, pos, rq);
                    const float dist = fmaf(-(2.0F * x->g1[pos]), s, d2 + x->h3[pos]);
                    const uint32_t id = x->ids[pos];
                    if (cnt < k) { /* sift up */
                        size_t i = cnt++;
                        hd[i] = dist; hi[i] = id;
                        while (i > 0) {
                            const size_t par = (i - 1) / 2;
                            if (!better(hd[par], hi[par], hd[i], hi[i])) break;
                            float td = hd[i]; hd[i] = hd[par]; hd[par] = td;
                            uint32_t ti = hi[i]; hi[i] = hi[par]; hi[par] = ti;
                            i = par;
                        }
                    } else if (better(dist, id, hd[0], hi[0])) {
                        hd[0] = dist; hi[0] = id;
                        size_t i = 0;
                        for (;;) {
                            const size_t l = 2 * i + 1, r = l + 1;
                            size_t lg = i;
                            if (l < k && better(hd[lg], hi[lg], hd[l], hi[l])) lg = l;
                            if (r < k && better(hd[lg], hi[lg], hd[r], hi[r])) lg = r;
                            if (lg == i) break;
                            float td = hd[i]; hd[i] = hd[lg]; hd[lg] = td;
                            uint32_t ti = hi[i]; hi[i] = hi[lg]; hi[lg] = ti;
                            i = lg;
                        }
                    }
                }
            }
            /* sorted extraction by Better (selection sort; k <= 128) */
            uint32_t* oid = out_ids + (size_t)qi * k;
            float* od = out_dists + (size_t)qi * k;
            for (size_t j = 0; j < k; ++j) {
                if (j < cnt) {
                    size_t bi = j;
                    for (size_t t = j + 1; t < cnt; ++t)
                        if (better(hd[t], hi[t], hd[bi], hi[bi])) bi = t;
                    float td = hd[j]; hd[j] = hd[bi]; hd[bi] = td;
                    uint32_t ti = hi[j]; hi[j] = hi[bi]; hi[bi] = ti;
                    oid[j] = hi[j];
                    od[j] = hd[j];
                } else {
                    oid[j] = UINT32_MAX;
                    od[j] = INFINITY;
                }
            }
        }
        free(rq); free(probes); free(pd2); free(hd); free(hi);
    }
}

/* ------------------------------------------------------------------------
 * Pruned production path: PrepareQuery (src/index/e8q_search.cpp:20-73),
 * ScanClusterAvx512 (src/simd/e8q_search_avx512.cpp:552-751), CollectLanes
 * and OrthoBatchHeader (src/index/e8q_scan_common.hpp:86-156),
 * FlushSurvivors / RefineRowsAvx512 (e8q_search.cpp:182-207,
 * e8q_search_avx512.cpp:118-347), WriteOrthoBanks (e8q_build.cpp:31-80).
 * Scalar expressions that the reference's GCC build contracts into fused
 * multiply-adds are spelled with fmaf(); the vector intrinsics' fmadd /
 * fnmadd are fmaf() by definition.
 * ---------------------------------------------------------------------- */

double orc_phi_inv(double p) {
    if (p <= 0.0) return -8.0;
    if (p >= 1.0) return 8.0;
    const double t = p < 1.0 - p ? p : 1.0 - p;
    double x = sqrt(-2.0 * log(t));
    if (p < 0.5) x = -x;
    for (int it = 0; it < 12; ++it) {
        const double phi = 0.3989422804014327 * exp(-0.5 * x * x);
        const double Phi = 0.5 * (1.0 + erf(x * 0.7071067811865476));
        x -= (Phi - p) / phi;
    }
    return x;
}

float orc_ortho_quantile(double alpha, size_t k_eff) {
    double tail = alpha / (double)(k_eff > 1 ? k_eff : 1);
    if (tail > 0.49) tail = 0.49;
    const double z = orc_phi_inv(1.0 - tail);
    return (float)(z > 1.0 ? z : 1.0);
}

static int clamp_u8(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }

void orc_ortho_header(const float* base, const float* weight, const float* perp, size_t cnt,
                      uint8_t* hdr) {
    float bmin = 0.0F, bmax = 0.0F, wmin = 0.0F, wmax = 0.0F, pmin = 0.0F, pmax = 0.0F;
    if (cnt > 0) {
        bmin = bmax = base[0];
        wmin = wmax = weight[0];
        pmin = pmax = perp[0];
        for (size_t i = 1; i < cnt; ++i) {
            if (base[i] < bmin) bmin = base[i];
            if (base[i] > bmax) bmax = base[i];
            if (weight[i] < wmin) wmin = weight[i];
            if (weight[i] > wmax) wmax = weight[i];
            if (perp[i] < pmin) pmin = perp[i];
            if (perp[i] > pmax) pmax = perp[i];
        }
    }
    const float wamax = fabsf(wmin) > fabsf(wmax) ? fabsf(wmin) : fabsf(wmax);
    const float bsc = bmax > bmin ? (bmax - bmin) / 255.0F : 1.0F;
    const float wsc = wmax > wmin ? (wmax - wmin) / 255.0F : 1.0F;
    const float psc = pmax > pmin ? (pmax - pmin) / 255.0F : 1.0F;
    memset(hdr, 0, 128);
    for (size_t i = 0; i < cnt; ++i) {
        hdr[i] = (uint8_t)clamp_u8((int)((base[i] - bmin) / bsc));          /* truncation */
        hdr[32 + i] = (uint8_t)clamp_u8((int)lroundf((weight[i] - wmin) / wsc)); /* nearest */
        hdr[64 + i] = (uint8_t)clamp_u8((int)ceilf((perp[i] - pmin) / psc));   /* up */
    }
    const float sc[7] = {bmin, bsc, wmin, wsc, pmin, psc, wamax};
    memcpy(hdr + 96, sc, sizeof(sc));
}

size_t orc_e8q_banks(const orc_e8q_index* x, uint8_t* out) {
    size_t nb = 0;
    float ob[32], ow[32], op[32];
    for (size_t c = 0; c < x->nlist; ++c) {
        const uint64_t lo = x->list_begin[c], hi = x->list_begin[c + 1];
        for (uint64_t b0 = lo; b0 < hi; b0 += 32, ++nb) {
            if (!out) continue;
            const size_t cnt = (size_t)(hi - b0 < 32 ? hi - b0 : 32);
            for (size_t i = 0; i < cnt; ++i) {
                ob[i] = x->ortho[(b0 + i) * 3 + 0];
                ow[i] = x->ortho[(b0 + i) * 3 + 1];
                op[i] = x->ortho[(b0 + i) * 3 + 2];
            }
            orc_ortho_header(ob, ow, op, cnt, out + nb * 128);
        }
    }
    return nb;
}

uint8_t orc_e8q_rowa(const orc_e8q_index* x, size_t pos, int blk) {
    return orc_pack_coarse(x->digits + (pos * (size_t)x->blocks + (size_t)blk) * 8,
                           x->branch[pos * (size_t)x->blocks + (size_t)blk], x->bits);
}

void orc_e8q_prepare_lut(int bits, int blocks, const float* rq, uint8_t* lut, float* scal) {
    /* gate_mid_: InitBitTables, src/index/e8q_io.cpp:213-228 */
    double w_cls[2], mid[16];
    orc_scan_class_means(bits, w_cls);
    for (int d = 0; d < 8; ++d) {
        mid[2 * d] = (bits == 1 && d == 7) ? 0.0 : w_cls[0];
        mid[2 * d + 1] = (bits == 1 && d == 7) ? 0.0 : w_cls[1];
    }
    float* cf = (float*)malloc(sizeof(float) * (size_t)blocks * 32);
    float hc = 0.0F;
    for (int blk = 0; blk < blocks; ++blk) {
        const float* qb = rq + (size_t)blk * 8;
        float* A = cf + (size_t)blk * 32; /* prices the low nibble: digits 4..7 */
        float* Bt = A + 16;               /* the high nibble: digits 0..3 */
        for (int v = 0; v < 16; ++v) {
            double av = 0.0, bv = 0.0;
            for (int h = 0; h < 4; ++h) {
                const int bit = (v >> (3 - h)) & 1;
                av = fma((double)qb[4 + h], mid[2 * (4 + h) + bit], av);
                bv = fma((double)qb[h], mid[2 * h + bit], bv);
            }
            A[v] = (float)av;
            Bt[v] = (float)bv;
        }
    }
    for (size_t i = 0; i < (size_t)blocks * 32; ++i)
        if (fabsf(cf[i]) > hc) hc = fabsf(cf[i]);
    const float delta = hc > 0.0F ? 2.0F * hc / 255.0F : 1.0F;
    const float qinv = 1.0F / delta, qoff = hc / delta;
    /* QuantizeU8Avx512: cvtps_epi32 (round to nearest even) of
     * fmadd(x, qinv, qoff), then unsigned saturation to u8 */
    for (size_t i = 0; i < (size_t)blocks * 32; ++i) {
        const int v = (int)nearbyintf(fmaf(cf[i], qinv, qoff));
        const uint32_t u = (uint32_t)v;
        lut[i] = (uint8_t)(u > 255u ? 255u : u);
    }
    free(cf);
    const float sqrt_blocks = sqrtf((float)blocks);
    scal[0] = delta;
    scal[1] = -hc * (float)(2 * blocks);
    scal[2] = 2.0F * sqrt_blocks * delta; /* LutErrClt */
    scal[3] = (float)blocks * fmaf(255.0F, delta, 2.0F * hc);
    (void)bits;
}

int32_t orc_e8q_coarse(const orc_e8q_index* x, size_t pos, const uint8_t* lut) {
    int32_t acc = 0;
    for (int blk = 0; blk < x->blocks; ++blk) {
        const uint8_t h = pos == (size_t)-1 ? 0 : orc_e8q_rowa(x, pos, blk);
        acc += lut[blk * 32 + (h & 0xF)] + lut[blk * 32 + 16 + (h >> 4)];
    }
    return acc;
}

float orc_e8q_refine_score(const orc_e8q_index* x, size_t pos, const float* rq) {
    const uint16_t* dg = x->digits + pos * (size_t)x->blocks * 8;
    const uint8_t* br = x->branch + pos * (size_t)x->blocks;
    float acc[8] = {0}, acc2[8] = {0};
    for (int blk = 0; blk < x->blocks; ++blk) {
        const float* tab = x->tab + (size_t)br[blk] * (size_t)x->tab_stride;
        float* dst = (blk & 1) ? acc2 : acc;
        for (int d = 0; d < 8; ++d) dst[d] = fmaf(tab[dg[blk * 8 + d]], rq[blk * 8 + d], dst[d]);
    }
    float t[8], s4[4];
    for (int d = 0; d < 8; ++d) t[d] = acc[d] + acc2[d];
    for (int i = 0; i < 4; ++i) s4[i] = t[i] + t[i + 4];
    const float s2a = s4[0] + s4[2], s2b = s4[1] + s4[3];
    return s2a + s2b;
}

typedef struct {
    size_t pos;
    float g1, h3; /* h3 = d2 + h3 of the row */
} orc_row;

typedef struct {
    float* hd;
    uint32_t* hi;
    size_t k, cnt;
} orc_heap;

/* InsertHeap: src/index/e8q_search.cpp:135-180 */
static void heap_insert(orc_heap* h, float dist, uint32_t id) {
    if (h->cnt < h->k) {
        size_t i = h->cnt++;
        h->hd[i] = dist;
        h->hi[i] = id;
        while (i > 0) {
            const size_t par = (i - 1) / 2;
            if (!better(h->hd[par], h->hi[par], h->hd[i], h->hi[i])) break;
            float td = h->hd[i]; h->hd[i] = h->hd[par]; h->hd[par] = td;
            uint32_t ti = h->hi[i]; h->hi[i] = h->hi[par]; h->hi[par] = ti;
            i = par;
        }
        return;
    }
    if (!better(dist, id, h->hd[0], h->hi[0])) return;
    h->hd[0] = dist;
    h->hi[0] = id;
    size_t i = 0;
    for (;;) {
        const size_t l = 2 * i + 1, r = l + 1;
        size_t lg = i;
        if (l < h->k && better(h->hd[lg], h->hi[lg], h->hd[l], h->hi[l])) lg = l;
        if (r < h->k && better(h->hd[lg], h->hi[lg], h->hd[r], h->hi[r])) lg = r;
        if (lg == i) break;
        float td = h->hd[i]; h->hd[i] = h->hd[lg]; h->hd[lg] = td;
        uint32_t ti = h->hi[i]; h->hi[i] = h->hi[lg]; h->hi[lg] = ti;
        i = lg;
    }
}

static float heap_limit(const orc_heap* h) { return h->cnt == h->k ? h->hd[0] : INFINITY; }

static void flush_rows(const orc_e8q_index* x, orc_row* rows, size_t* n, const float* rq,
                       orc_heap* h) {
    for (size_t j = 0; j < *n; ++j) {
        const float s = orc_e8q_refine_score(x, rows[j].pos, rq);
        heap_insert(h, fmaf(-(2.0F * rows[j].g1), s, rows[j].h3), x->ids[rows[j].pos]);
    }
    *n = 0;
}

void orc_e8q_search_pruned(const orc_e8q_index* x, const uint8_t* banks_in, float alpha,
                           int disable_prune, const float* queries, size_t nq, size_t k,
                           size_t nprobe, uint32_t* out_ids, float* out_dists, uint64_t* cand_out,
                           uint64_t* surv_out, int threads) {
    const size_t nbatches = orc_e8q_banks(x, NULL);
    uint8_t* own = NULL;
    const uint8_t* banks = banks_in;
    if (!banks) {
        own = (uint8_t*)malloc(nbatches * 128 + 1);
        orc_e8q_banks(x, own);
        banks = own;
    }
    /* first batch of each list */
    size_t* bfirst = (size_t*)malloc(sizeof(size_t) * (x->nlist + 1));
    bfirst[0] = 0;
    for (size_t c = 0; c < x->nlist; ++c)
        bfirst[c + 1] = bfirst[c] + (size_t)((x->list_begin[c + 1] - x->list_begin[c] + 31) / 32);
    const size_t k_eff = 4 * k > 32 ? 4 * k : 32;
    const float z = orc_ortho_quantile((double)alpha, k_eff);
    const int B = x->blocks;
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        float* rq = (float*)malloc(sizeof(float) * x->padded_dim);
        uint32_t* probes = (uint32_t*)malloc(sizeof(uint32_t) * x->nlist);
        float* pd2 = (float*)malloc(sizeof(float) * x->nlist);
        uint8_t* lut = (uint8_t*)malloc((size_t)B * 32);
        orc_heap h;
        h.hd = (float*)malloc(sizeof(float) * (k + 1));
        h.hi = (uint32_t*)malloc(sizeof(uint32_t) * (k + 1));
        h.k = k;
        orc_row rows[32];
#pragma omp for schedule(dynamic, 1)
        for (long long qi = 0; qi < (long long)nq; ++qi) {
            float scal[4];
            orc_e8q_prepare_query(x, queries + (size_t)qi * x->dim, rq);
            orc_e8q_prepare_lut(x->bits, B, rq, lut, scal);
            const float delta_c = scal[0], base_c = scal[1], lut_err = scal[2], score_max = scal[3];
            const size_t take = nprobe < x->nlist ? nprobe : x->nlist;
            orc_e8q_route(x, rq, take, probes, pd2);
            const int32_t pad_acc = orc_e8q_coarse(x, (size_t)-1, lut);
            h.cnt = 0;
            size_t nst = 0;
            uint64_t cand = 0, surv = 0;
            for (size_t p = 0; p < take; ++p) {
                const size_t c = probes[p];
                const float d2 = pd2[p];
                const uint64_t lo = x->list_begin[c], cnt = x->list_begin[c + 1] - lo;
                if (cnt == 0) continue;
                const float sqrt_d2 = sqrtf(d2 > 0.0F ? d2 : 0.0F);
                for (uint64_t off = 0; off < cnt; off += 32) {
                    const size_t n_logic = (size_t)(cnt - off < 32 ? cnt - off : 32);
                    const uint8_t* bp = banks + (bfirst[c] + (size_t)(off / 32)) * 128;
                    int32_t accC[32];
                    for (size_t t = 0; t < 32; ++t)
                        accC[t] = t < n_logic ? orc_e8q_coarse(x, (size_t)(lo + off + t), lut) : pad_acc;
                    cand += n_logic;
                    const float distk0 = heap_limit(&h);
                    const float r_horizon =
                        (distk0 < d2) ? sqrtf(distk0 > 0.0F ? distk0 : 0.0F) : sqrt_d2;
                    float sc[7];
                    memcpy(sc, bp + 96, sizeof(sc));
                    const float base_min = sc[0], base_scale = sc[1], wmin = sc[2], wscale = sc[3];
                    const float perp_min = sc[4], perp_scale = sc[5];
                    const float pad_w_lut = lut_err;
                    const float pad_w_round = 0.5F * wscale * (score_max + lut_err);
                    if (!disable_prune && distk0 < INFINITY) {
                        /* whole-batch skip (:611-635) */
                        const float w_amax = sc[6];
                        const float pad_add = fmaf(w_amax, pad_w_lut, pad_w_round);
                        const float perp_amax = fmaf(255.0F, perp_scale, perp_min);
                        int32_t mx = accC[0], mn = accC[0];
                        for (int t = 1; t < 32; ++t) {
                            if (accC[t] > mx) mx = accC[t];
                            if (accC[t] < mn) mn = accC[t];
                        }
                        const float s_hi = fmaf((float)mx, delta_c, base_c);
                        const float s_lo = fmaf((float)mn, delta_c, base_c);
                        const float s_absmax = fabsf(s_hi) > fabsf(s_lo) ? fabsf(s_hi) : fabsf(s_lo);
                        const float lb = fmaf(-(z * r_horizon), perp_amax,
                                              fmaf(-w_amax, s_absmax, (d2 + base_min) - pad_add));
                        if (lb >= distk0) continue;
                    }
                    /* per-lane bound (:636-676) */
                    float dlo[32];
                    const float bmin_d2 = (base_min + d2) - pad_w_round;
                    const float slack = z * r_horizon;
                    for (int t = 0; t < 32; ++t) {
                        const float scv = fmaf((float)accC[t], delta_c, base_c);
                        const float base_term = fmaf((float)bp[t], base_scale, bmin_d2);
                        const float weight = fmaf((float)bp[32 + t], wscale, wmin);
                        const float perp = fmaf((float)bp[64 + t], perp_scale, perp_min);
                        const float dc = fmaf(-weight, scv, base_term);
                        dlo[t] = fmaf(-slack, perp, fmaf(-fabsf(weight), pad_w_lut, dc));
                    }
                    uint32_t mask = 0;
                    if (disable_prune) {
                        mask = 0xFFFFFFFFu;
                    } else {
                        for (int t = 0; t < 32; ++t)
                            if (dlo[t] < distk0) mask |= 1u << t;
                    }
                    if (n_logic < 32) mask &= (1u << n_logic) - 1u;
                    /* CollectLanes (e8q_scan_common.hpp:86-113) */
                    while (mask) {
                        const int lane = __builtin_ctz(mask);
                        mask &= mask - 1;
                        if (!disable_prune && !(dlo[lane] < heap_limit(&h))) continue;
                        if (nst >= 32) flush_rows(x, rows, &nst, rq, &h);
                        ++surv;
                        const size_t pos = (size_t)(lo + off) + (size_t)lane;
                        rows[nst].pos = pos;
                        rows[nst].g1 = x->g1[pos];
                        rows[nst].h3 = d2 + x->h3[pos];
                        ++nst;
                    }
                }
                flush_rows(x, rows, &nst, rq, &h);
            }
            flush_rows(x, rows, &nst, rq, &h);
            /* ExtractTopK: src/index/e8q_search.cpp:295-318 */
            uint32_t* oid = out_ids + (size_t)qi * k;
            float* od = out_dists + (size_t)qi * k;
            for (size_t j = 0; j < k; ++j) {
                if (j < h.cnt) {
                    size_t bi = j;
                    for (size_t t = j + 1; t < h.cnt; ++t)
                        if (better(h.hd[t], h.hi[t], h.hd[bi], h.hi[bi])) bi = t;
                    float td = h.hd[j]; h.hd[j] = h.hd[bi]; h.hd[bi] = td;
                    uint32_t ti = h.hi[j]; h.hi[j] = h.hi[bi]; h.hi[bi] = ti;
                    oid[j] = h.hi[j];
                    od[j] = h.hd[j];
                } else {
                    oid[j] = 0xFFFFFFFFu;
                    od[j] = INFINITY;
                }
            }
            if (cand_out) cand_out[qi] = cand;
            if (surv_out) surv_out[qi] = surv;
        }
        free(rq); free(probes); free(pd2); free(lut); free(h.hd); free(h.hi);
    }
    free(bfirst);
    free(own);
}


/* ProbeBoundW: src/index/e8q_oracle.cpp:103-218. Query and base row are
 * rotated and centred like the build's rows; the exact reconstruction uses
 * the double level tables / sqrt(Dpad) and the scan basis the class means of
 * InitBitTables (src/index/e8q_io.cpp:213-228: zero for dim 7 at 1 bit).
 * The reference decodes each block with the 8-bit-digit split decoder
 * (e8q_oracle.cpp:177-184 calls DecodeSplitBlockLane with uint8_t digits,
 * src/index/e8q_scan.cpp:34-60), and this restates what that returns from the
 * stored digits: at 2..8 bits the real digits and branch; at 1 bit the refine
 * field is empty, so digit 7 is the rowA byte's bit 0 (the branch) and the
 * branch reads 0; at 9 bits the digits keep their low 8 bits (the top bit
 * falls out of the uint8_t). Above 9 bits the reference's decoder copies more
 * than its 8-byte staging integer holds; the same low-8-bit rule is used. */
static void probe_digits(int bits, const uint16_t* real, int branch, int* dg, int* br) {
    for (int k = 0; k < 8; ++k) dg[k] = real[k];
    *br = branch;
    if (bits == 1) {
        dg[7] = branch;
        *br = 0;
    } else if (bits >= 9) {
        for (int k = 0; k < 8; ++k) dg[k] &= 0xFF;
    }
}

double orc_e8q_probe_bound_w(const orc_e8q_index* x, const float* q, const float* base_row, uint32_t id) {
    size_t pos = (size_t)-1;
    for (size_t i = 0; i < x->n; ++i)
        if (x->ids[i] == id) { pos = i; break; }
    if (pos == (size_t)-1) return NAN;
    const size_t c = list_of(x, pos);
    const size_t pd = x->padded_dim;
    const float* cc = x->centroid_rot + c * pd;
    float* rq = (float*)malloc(sizeof(float) * pd);
    float* rx = (float*)malloc(sizeof(float) * pd);
    double* unit = (double*)malloc(sizeof(double) * pd);
    orc_e8q_prepare_query(x, q, rq);
    orc_e8q_prepare_query(x, base_row, rx);
    double d2 = 0.0, rn2 = 0.0;
    for (size_t d = 0; d < pd; ++d) {
        const double qr = (double)rq[d] - (double)cc[d];
        const double xr = (double)rx[d] - (double)cc[d];
        d2 += qr * qr;
        rn2 += xr * xr;
        unit[d] = xr;
    }
    const double rn = sqrt(rn2);
    double out = NAN;
    if (rn > 0.0) {
        for (size_t d = 0; d < pd; ++d) unit[d] /= rn;
        const int bits = x->bits, qn = 1 << bits;
        double* lev = (double*)malloc(sizeof(double) * 2 * (size_t)qn);
        orc_branch_levels(bits, 0, lev);
        orc_branch_levels(bits, 1, lev + qn);
        double w_cls[2], mid[16];
        orc_scan_class_means(bits, w_cls);
        for (int d = 0; d < 8; ++d) {
            mid[2 * d] = (bits == 1 && d == 7) ? 0.0 : w_cls[0];
            mid[2 * d + 1] = (bits == 1 && d == 7) ? 0.0 : w_cls[1];
        }
        const double rd = sqrt((double)pd);
        double dot_ue = 0, n2_e = 0, dot_ce = 0, dot_ew = 0, dot_uw = 0, n2_w = 0, dot_cw = 0, s_exact = 0,
               s_coarse = 0;
        const uint16_t* dg = x->digits + pos * (size_t)x->blocks * 8;
        const uint8_t* br = x->branch + pos * (size_t)x->blocks;
        for (int blk = 0; blk < x->blocks; ++blk) {
            int pdg[8], pbr = 0;
            probe_digits(bits, dg + (size_t)blk * 8, br[blk], pdg, &pbr);
            for (int k = 0; k < 8; ++k) {
                const size_t idx = (size_t)blk * 8 + (size_t)k;
                const int g = pdg[k];
                const double ve = lev[(size_t)pbr * (size_t)qn + (size_t)g] / rd;
                const double wc = mid[2 * k + (g >> (bits - 1))];
                dot_ue += unit[idx] * ve;
                n2_e += ve * ve;
                dot_ce += (double)cc[idx] * ve;
                dot_ew += ve * wc;
                dot_uw += unit[idx] * wc;
                n2_w += wc * wc;
                dot_cw += (double)cc[idx] * wc;
                s_exact += (double)rq[idx] * ve;
                s_coarse += (double)rq[idx] * wc;
            }
        }
        free(lev);
        if (fabs(dot_ue) > 0.0 && fabs(dot_uw) > 0.0) {
            const double g1 = rn / dot_ue;
            const double h3 = rn2 + 2.0 * g1 * dot_ce;
            const double d_full = d2 + h3 - 2.0 * g1 * s_exact;
            const double w_x = 2.0 * rn / dot_uw;
            const double d_coarse = d2 + rn2 + w_x * dot_cw - w_x * s_coarse;
            const double rx2 = 4.0 * g1 * g1 * n2_e + w_x * w_x * n2_w - 4.0 * g1 * w_x * dot_ew;
            const double sqrt_dm1 = sqrt((double)(x->dim > 1 ? x->dim - 1 : 1));
            const double omega = sqrt(rx2 > 0.0 ? rx2 : 0.0) / sqrt_dm1;
            const double r_q = sqrt(d2 > 0.0 ? d2 : 0.0);
            if (omega > 0.0 && r_q > 0.0) out = (d_coarse - d_full) / (r_q * omega);
        }
    }
    free(rq);
    free(rx);
    free(unit);
    return out;
}
