// Host-side codec constants: companded level tables, the per-rate scale
// schedule and the sorted search tables the GPU encoder walks.
//
// Compiled with -ffp-contract=off. The reference's GCC build contracts the
// Horner steps of the inverse-normal approximation into fused multiply-adds
// (C++ default fp-contract=fast with an FMA -march), and the level values,
// hence the codes, depend on that; the steps are therefore written as
// std::fma and nothing else may be fused.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "internal.h"

namespace e8qc {

// Acklam's rational approximation of the inverse normal CDF (P. J. Acklam,
// 2003; published coefficients): src/quantization/e8q_codec.cpp:17-44.
double inv_normal_cdf(double p) {
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
    auto tail = [&](double q) {
        const double num =
            std::fma(std::fma(std::fma(std::fma(std::fma(c[0], q, c[1]), q, c[2]), q, c[3]), q,
                              c[4]),
                     q, c[5]);
        const double den =
            std::fma(std::fma(std::fma(std::fma(d[0], q, d[1]), q, d[2]), q, d[3]), q, 1.0);
        return num / den;
    };
    if (p < plow) return tail(std::sqrt(-2 * std::log(std::max(p, 1e-300))));
    if (p <= 1 - plow) {
        const double q = p - 0.5;
        const double r = q * q;
        const double num =
            std::fma(std::fma(std::fma(std::fma(std::fma(a[0], r, a[1]), r, a[2]), r, a[3]), r,
                              a[4]),
                     r, a[5]) *
            q;
        const double den =
            std::fma(std::fma(std::fma(std::fma(std::fma(b[0], r, b[1]), r, b[2]), r, b[3]), r,
                              b[4]),
                     r, 1.0);
        return num / den;
    }
    return -tail(std::sqrt(-2 * std::log(std::max(1 - p, 1e-300))));
}

// Digit d = t mod q carries the quantile 1/2 + (t + eta)/q, eta = 1/4 or 3/4
// by branch: src/quantization/e8q_codec.cpp:496-509.
std::vector<double> branch_levels(int bits, int branch) {
    const int q = 1 << bits;
    const double eta = 0.25 + 0.5 * static_cast<double>(branch);
    std::vector<double> out(static_cast<size_t>(q));
    const int start = static_cast<int>(std::ceil(-0.5 * static_cast<double>(q) - eta));
    for (int i = 0; i < q; ++i) {
        const long t = static_cast<long>(start + i);
        const int digit = static_cast<int>(((t % q) + q) % q);
        const double p = 0.5 + (static_cast<double>(t) + eta) / static_cast<double>(q);
        out[static_cast<size_t>(digit)] =
            kSigmaC * inv_normal_cdf(std::min(1.0 - 1e-12, std::max(1e-12, p)));
    }
    return out;
}

// Per-rate encoding scale: the constant schedule the reference fixes at
// src/quantization/e8q_codec.cpp:456-460 (codes depend on it).
double fixed_scale(int bits) {
    static const double sched[kMaxBits + 1] = {0.0,   1.118034, 0.895, 0.825, 0.785,
                                               0.755, 0.735,    0.735, 0.735, 0.725,
                                               0.715, 0.705,    0.710, 0.705};
    return sched[std::min(std::max(bits, 1), kMaxBits)];
}

// Newton on Phi from the asymptotic start, 12 steps (std::erf / std::exp /
// std::log, the functions the reference calls): src/index/e8q_internal.hpp:75-97.
double phi_inv(double p) {
    if (p <= 0.0) return -8.0;
    if (p >= 1.0) return 8.0;
    const double t = std::min(p, 1.0 - p);
    double x = std::sqrt(-2.0 * std::log(t));
    if (p < 0.5) x = -x;
    for (int it = 0; it < 12; ++it) {
        const double phi = 0.3989422804014327 * std::exp(-0.5 * x * x);
        const double Phi = 0.5 * (1.0 + std::erf(x * 0.7071067811865476));
        x -= (Phi - p) / phi;
    }
    return x;
}

// src/index/e8q_internal.hpp:99-107.
float ortho_quantile(double alpha, size_t k_eff) {
    const double tail = std::min(alpha / static_cast<double>(std::max<size_t>(k_eff, 1)), 0.49);
    return static_cast<float>(std::max(phi_inv(1.0 - tail), 1.0));
}

namespace {

// Bounded-bin index (src/quantization/e8q_codec.cpp:70-123): bins no wider
// than the tightest level gap, usable only when every bin holds <= 2 levels.
void build_bin_index(LevelTableHost& t, int max_bins) {
    const double* lev = t.lev.data() + t.pad;
    const int n = t.n;
    t.usable = 0;
    t.bin_lo.clear();
    if (n < 16) return;
    const double lo = lev[0], hi = lev[n - 1];
    if (!(hi > lo)) return;
    double min_gap = DBL_MAX;
    for (int i = 1; i < n; ++i) min_gap = std::min(min_gap, lev[i] - lev[i - 1]);
    if (!(min_gap > 0.0)) return;
    const double range = hi - lo;
    long bins = 1;
    while (static_cast<double>(bins) * min_gap < range && bins < max_bins) bins *= 2;
    if (static_cast<double>(bins) * min_gap < range) return;
    t.nbins = static_cast<int>(bins);
    t.bin_lo_v = lo;
    t.bin_scale = static_cast<double>(bins) / range;
    t.bin_lo.assign(static_cast<size_t>(bins) + 1, 0);
    int j = 0;
    for (long b = 0; b <= bins; ++b) {
        const double edge = lo + static_cast<double>(b) / t.bin_scale;
        while (j < n && lev[j] < edge) ++j;
        t.bin_lo[static_cast<size_t>(b)] = static_cast<uint32_t>(j);
    }
    int max_span = 0;
    for (long b = 0; b < bins; ++b)
        max_span = std::max(max_span, static_cast<int>(t.bin_lo[b + 1] - t.bin_lo[b]));
    t.usable = max_span <= 2;
}

EncTablesHost make_tables(int bits) {
    EncTablesHost et;
    et.bits = bits;
    et.levels[0] = branch_levels(bits, 0);
    et.levels[1] = branch_levels(bits, 1);
    const int q = 1 << bits;
    const int n = 2 * q;
    // Merged table: sorted union of both branches' levels
    // (src/quantization/e8q_codec.cpp:297-352); stable by (value, branch-0-first
    // insertion order). Class r = 2*parity + branch sits at positions i with
    // (i & 3) == r when the interleaving holds.
    struct Ent {
        double v;
        uint16_t dig;
        uint8_t br;
    };
    std::vector<Ent> raw;
    raw.reserve(static_cast<size_t>(n));
    for (int d = 0; d < q; ++d) {
        raw.push_back({et.levels[0][d], static_cast<uint16_t>(d), 0});
        raw.push_back({et.levels[1][d], static_cast<uint16_t>(d), 1});
    }
    std::stable_sort(raw.begin(), raw.end(), [](const Ent& a, const Ent& b) { return a.v < b.v; });
    bool alt = true;
    for (int i = 0; i < n && alt; ++i) {
        if (i > 0 && !(raw[i].v > raw[i - 1].v)) alt = false;
        if (raw[i].br != static_cast<uint8_t>(i & 1) ||
            (raw[i].dig & 1u) != static_cast<unsigned>((i >> 1) & 1))
            alt = false;
    }
    et.alternating = alt ? 1 : 0;
    LevelTableHost& m = et.merged;
    m.pad = 4;
    m.n = n;
    m.lev.assign(static_cast<size_t>(n) + 8, INFINITY);
    m.dig.assign(static_cast<size_t>(n) + 8, 0);
    for (int i = 0; i < 4; ++i) m.lev[i] = -INFINITY;
    for (int i = 0; i < n; ++i) {
        m.lev[4 + i] = raw[i].v;
        m.dig[4 + i] = raw[i].dig;
    }
    if (alt) build_bin_index(m, 32768);
    // Per-(branch, parity) tables (src/quantization/e8q_codec.cpp:142-186):
    // sorted by (level, digit), two +inf pads.
    for (int br = 0; br < 2; ++br) {
        for (int odd = 0; odd < 2; ++odd) {
            LevelTableHost& t = et.parity[br][odd];
            std::vector<std::pair<double, uint16_t>> e;
            for (int d = odd; d < q; d += 2) e.push_back({et.levels[br][d], static_cast<uint16_t>(d)});
            std::stable_sort(e.begin(), e.end(), [](const auto& a, const auto& b) {
                return a.first < b.first || (a.first == b.first && a.second < b.second);
            });
            t.pad = 0;
            t.n = static_cast<int>(e.size());
            t.lev.resize(e.size() + 2);
            t.dig.assign(e.size() + 2, 0);
            for (size_t i = 0; i < e.size(); ++i) {
                t.lev[i] = e[i].first;
                t.dig[i] = e[i].second;
            }
            t.lev[e.size()] = INFINITY;
            t.lev[e.size() + 1] = INFINITY;
            build_bin_index(t, 16384);
        }
    }
    return et;
}

}  // namespace

const EncTablesHost& enc_tables_host(int bits) {
    static std::mutex mu;
    static std::map<int, EncTablesHost> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(bits);
    if (it == cache.end()) it = cache.emplace(bits, make_tables(bits)).first;
    return it->second;
}

namespace {
template <class T>
T* upload(const std::vector<T>& v) {
    T* p = nullptr;
    const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
    E8QC_CUDA(cudaMalloc(&p, bytes));
    if (!v.empty()) E8QC_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return p;
}

DevLevelTable upload_table(const LevelTableHost& t) {
    DevLevelTable d{};
    const double* lev = upload(t.lev);
    const uint16_t* dig = upload(t.dig);
    d.lev = lev + t.pad;
    d.dig = dig + t.pad;
    d.bin_lo = upload(t.bin_lo);
    d.n = t.n;
    d.nbins = t.nbins;
    d.usable = t.usable;
    d.bin_lo_v = t.bin_lo_v;
    d.bin_scale = t.bin_scale;
    return d;
}
}  // namespace

const DevEncTables& enc_tables_device(int device, int bits) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, DevEncTables> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(device, bits);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const EncTablesHost& h = enc_tables_host(bits);
    DevEncTables d{};
    d.bits = bits;
    d.alternating = h.alternating;
    d.merged = upload_table(h.merged);
    for (int br = 0; br < 2; ++br)
        for (int odd = 0; odd < 2; ++odd) d.parity[br * 2 + odd] = upload_table(h.parity[br][odd]);
    d.levels[0] = upload(h.levels[0]);
    d.levels[1] = upload(h.levels[1]);
    return cache.emplace(key, d).first->second;
}

}  // namespace e8qc
