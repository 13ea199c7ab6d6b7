// pybind11 module `_e8qlib`: the reference's Python API (E8qIndex) over the
// C ABI of libe8qcuda.so.
//
// Same class, argument names, defaults, dtypes, shapes, padding values and
// exception types as python_bindings/e8q_bindings.cpp:22-344 of the
// reference: inputs are force-cast to C-contiguous float32 / uint32,
// std::invalid_argument -> ValueError, std::runtime_error -> RuntimeError.
// `num_threads` is accepted and ignored (the work runs on the GPU).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <cstdint>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "e8qc.h"

namespace py = pybind11;

namespace e8qb200 {

template <typename T>
py::array_t<T, py::array::c_style | py::array::forcecast> ensure_nd(py::handle v, const char* name,
                                                                    int nd) {
    auto a = py::array_t<T, py::array::c_style | py::array::forcecast>::ensure(v);
    if (!a) throw std::invalid_argument(std::string(name) + " must be a NumPy array");
    if (a.ndim() != nd)
        throw std::invalid_argument(std::string(name) + (nd == 2 ? " must be a 2D NumPy array"
                                                                 : " must be a 1D NumPy array"));
    return a;
}

// Status code -> the exception type the reference raises for that condition.
void check(int rc) {
    if (rc == E8QC_OK) return;
    const std::string msg = e8qc_last_error();
    switch (rc) {
        case E8QC_EINVAL:
        case E8QC_ERANGE: throw std::invalid_argument(msg);
        case E8QC_ENOMEM: throw std::runtime_error("out of memory: " + msg);
        default: throw std::runtime_error(msg);
    }
}

int mode_of(const std::string& m) {
    if (m == "plain") return E8QC_MODE_PLAIN;
    if (m == "batched") return E8QC_MODE_BATCHED;
    if (m == "precision") return E8QC_MODE_PRECISION;
    if (m == "pruned") return E8QC_MODE_PRUNED;
    throw std::invalid_argument("mode must be 'auto', 'plain', 'pruned', 'batched' or 'precision'");
}

// ME8Q search modes: the grouped exact scan, or int8 tensor-core candidates
// with exact rescoring.
int me8q_mode(const std::string& m) {
    if (m == "pruned") return E8QC_MODE_PRUNED;
    if (m == "batched") return E8QC_MODE_BATCHED;
    if (m == "precision") return E8QC_MODE_PRECISION;
    throw std::invalid_argument("ME8Q modes are 'pruned', 'batched' and 'precision'");
}

class E8qIndex {
   public:
    E8qIndex(size_t dim, size_t nbits, uint64_t seed, int device)
        : dim_(dim), nbits_(nbits), seed_(seed), device_(device) {
        if (dim == 0) throw std::invalid_argument("dim must be positive");
        if (nbits < 1 || nbits > 13) throw std::invalid_argument("nbits must be in [1, 13]");
    }
    ~E8qIndex() {
        if (idx_) e8qc_e8q_destroy(idx_);
    }
    E8qIndex(const E8qIndex&) = delete;
    E8qIndex& operator=(const E8qIndex&) = delete;

    void build(py::handle data, py::handle centroids, py::handle cluster_ids, size_t /*num_threads*/,
               float prune_alpha) {
        auto x = ensure_nd<float>(data, "data", 2);
        auto c = ensure_nd<float>(centroids, "centroids", 2);
        auto ids = ensure_nd<uint32_t>(cluster_ids, "cluster_ids", 1);
        if (static_cast<size_t>(x.shape(1)) != dim_)
            throw std::invalid_argument("data dimension does not match index dim");
        if (static_cast<size_t>(c.shape(1)) != dim_)
            throw std::invalid_argument("centroid dimension does not match index dim");
        if (ids.shape(0) != x.shape(0))
            throw std::invalid_argument("cluster_ids length must match number of rows in data");
        fresh();
        py::gil_scoped_release nogil;
        check(e8qc_e8q_build(idx_, x.data(), static_cast<size_t>(x.shape(0)), c.data(),
                             static_cast<size_t>(c.shape(0)), ids.data(), prune_alpha, nullptr));
        built_ = true;
    }

    // Device-resident build: raw CUDA pointers (e.g. torch tensor data_ptr()).
    void build_ptr(uintptr_t data, size_t n, uintptr_t centroids, size_t nlist, uintptr_t cluster_ids,
                   float prune_alpha, uintptr_t stream) {
        fresh();
        py::gil_scoped_release nogil;
        check(e8qc_e8q_build(idx_, reinterpret_cast<const float*>(data), n,
                             reinterpret_cast<const float*>(centroids), nlist,
                             reinterpret_cast<const uint32_t*>(cluster_ids), prune_alpha,
                             reinterpret_cast<void*>(stream)));
        built_ = true;
    }

    py::tuple search(py::handle queries, size_t k, size_t nprobe, size_t /*num_threads*/,
                     bool return_stats, const std::string& mode) {
        auto q = ensure_nd<float>(queries, "queries", 2);
        require("search");
        if (static_cast<size_t>(q.shape(1)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        if (k == 0) throw std::invalid_argument("k must be positive");
        if (k > E8QC_MAX_K) throw std::invalid_argument("k must be <= " + std::to_string(E8QC_MAX_K));
        if (nprobe == 0) throw std::invalid_argument("nprobe must be positive");
        const int md = search_mode(mode);
        const size_t nq = static_cast<size_t>(q.shape(0));
        py::array_t<uint32_t> ids({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k)});
        py::array_t<float> dists({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k)});
        uint32_t* ip = ids.mutable_data();
        float* dp = dists.mutable_data();
        std::fill(ip, ip + nq * k, std::numeric_limits<uint32_t>::max());
        std::fill(dp, dp + nq * k, std::numeric_limits<float>::infinity());
        e8qc_stats st{};
        {
            py::gil_scoped_release nogil;
            if (nq > 0) check(e8qc_e8q_search(idx_, q.data(), nq, k, nprobe, md, ip, dp,
                                              return_stats ? &st : nullptr, nullptr));
        }
        if (!return_stats) return py::make_tuple(ids, dists);
        return py::make_tuple(ids, dists, stats_dict(st, nq, nprobe));
    }

    // Device-resident search on raw CUDA pointers; returns the launch count.
    uint64_t search_ptr(uintptr_t queries, size_t nq, size_t k, size_t nprobe, uintptr_t out_ids,
                        uintptr_t out_dists, const std::string& mode, uintptr_t stream) {
        require("search");
        const int md = search_mode(mode);
        e8qc_stats st{};
        py::gil_scoped_release nogil;
        check(e8qc_e8q_search(idx_, reinterpret_cast<const float*>(queries), nq, k, nprobe, md,
                              reinterpret_cast<uint32_t*>(out_ids), reinterpret_cast<float*>(out_dists), &st,
                              reinterpret_cast<void*>(stream)));
        return st.launches;
    }

    // Serving form: per-query k and nprobe; rows padded to k_max.
    py::tuple search_ragged(py::handle queries, py::handle k, py::handle nprobe, size_t k_max,
                            const std::string& mode) {
        const int md = mode_of(mode);
        auto q = ensure_nd<float>(queries, "queries", 2);
        auto ka = ensure_nd<uint32_t>(k, "k", 1);
        auto na = ensure_nd<uint32_t>(nprobe, "nprobe", 1);
        require("search");
        if (static_cast<size_t>(q.shape(1)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        const size_t nq = static_cast<size_t>(q.shape(0));
        if (static_cast<size_t>(ka.shape(0)) != nq || static_cast<size_t>(na.shape(0)) != nq)
            throw std::invalid_argument("k and nprobe must have one entry per query");
        py::array_t<uint32_t> ids({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k_max)});
        py::array_t<float> dists({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k_max)});
        {
            py::gil_scoped_release nogil;
            if (nq > 0)
                check(e8qc_e8q_search_ragged_mode(idx_, q.data(), nq, ka.data(), na.data(), k_max, md,
                                                  ids.mutable_data(), dists.mutable_data(), nullptr, nullptr));
        }
        return py::make_tuple(ids, dists);
    }

    float estimate(py::handle query, uint32_t id) {
        require("estimate");
        auto q = ensure_nd<float>(query, "query", 1);
        if (static_cast<size_t>(q.shape(0)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        float out = 0.0f;
        check(e8qc_e8q_estimate(idx_, q.data(), id, &out));
        return out;
    }

    // "auto" is the reference's search: the pruned production path, or the
    // plain scan of every candidate after set_disable_prune(True).
    int search_mode(const std::string& mode) const {
        if (mode != "auto") return mode_of(mode);
        e8qc_info inf{};
        check(e8qc_e8q_info(idx_, &inf));
        return inf.disable_prune ? E8QC_MODE_PLAIN : E8QC_MODE_PRUNED;
    }

    // Thresholds of the last pruned search's first nq queries.
    py::array_t<float> pruned_thresholds(size_t nq) {
        require("pruned_thresholds");
        py::array_t<float> out(static_cast<py::ssize_t>(nq));
        check(e8qc_e8q_pruned_thresholds(idx_, out.mutable_data(), nq));
        return out;
    }

    // E8qIndex.probe_bound_w (e8q_bindings.cpp:182-233): the bound's
    // normalised discrepancy per (query, stored vector) pair, on the GPU.
    py::array_t<double> probe_bound_w(py::handle queries, py::handle base_rows, py::handle qidx, py::handle ids,
                                      size_t /*num_threads*/) {
        if (!built_ || idx_ == nullptr)
            throw std::runtime_error("E8qIndex must be built or loaded before probe_bound_w");
        auto q = ensure_nd<float>(queries, "queries", 2);
        auto b = ensure_nd<float>(base_rows, "base_rows", 2);
        auto qi = ensure_nd<uint32_t>(qidx, "qidx", 1);
        auto ii = ensure_nd<uint32_t>(ids, "ids", 1);
        if (static_cast<size_t>(q.shape(1)) != dim_)
            throw std::invalid_argument("queries dimension does not match index dim");
        if (static_cast<size_t>(b.shape(1)) != dim_)
            throw std::invalid_argument("base_rows dimension does not match index dim");
        const size_t m = static_cast<size_t>(ii.shape(0));
        if (static_cast<size_t>(qi.shape(0)) != m || static_cast<size_t>(b.shape(0)) != m)
            throw std::invalid_argument("qidx, ids and base_rows must have the same length");
        py::array_t<double> out(static_cast<py::ssize_t>(m));
        const size_t nq = static_cast<size_t>(q.shape(0));
        {
            py::gil_scoped_release nogil;
            check(e8qc_e8q_probe_bound_w(idx_, q.data(), nq, b.data(), qi.data(), ii.data(), m,
                                         out.mutable_data()));
        }
        return out;
    }

    // Fault injection (no reference counterpart): the next `searches` plain
    // searches give up a bounded device wait and raise (E8QC_ETIMEOUT).
    void debug_inject_wait_timeout(int searches, uint32_t wait_ms) {
        require("debug_inject_wait_timeout");
        check(e8qc_e8q_debug_inject_wait_timeout(idx_, searches, wait_ms));
    }

    void set_disable_prune(bool on) {
        require("set_disable_prune");
        check(e8qc_e8q_set_disable_prune(idx_, on ? 1 : 0));
    }
    void set_prune_alpha(float alpha) {
        require("set_prune_alpha");
        check(e8qc_e8q_set_prune_alpha(idx_, alpha));
    }

    py::tuple export_codes() {
        require("export_codes");
        const e8qc_info in = info();
        const size_t n = in.n, B = in.padded_dim / 8;
        py::array_t<uint32_t> ids(static_cast<py::ssize_t>(n));
        py::array_t<uint16_t> dg({static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(B), py::ssize_t(8)});
        py::array_t<uint8_t> br({static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(B)});
        py::array_t<float> g1(static_cast<py::ssize_t>(n)), h3(static_cast<py::ssize_t>(n));
        check(e8qc_e8q_get_ids(idx_, ids.mutable_data()));
        check(e8qc_e8q_export_codes(idx_, dg.mutable_data(), br.mutable_data(), g1.mutable_data(),
                                    h3.mutable_data()));
        return py::make_tuple(ids, dg, br, g1, h3);
    }

    py::dict autotune(const std::string& mode, size_t nq, size_t k, size_t nprobe) {
        require("autotune");
        e8qc_tuning t{};
        {
            py::gil_scoped_release nogil;
            check(e8qc_e8q_autotune(idx_, mode_of(mode), nq, k, nprobe, &t));
        }
        py::dict d;
        d["schedule"] = t.schedule == 0 ? "longest_list_first" : "list_id_order";
        d["stages"] = t.stages;
        d["best_ms"] = t.best_ms;
        d["default_ms"] = t.default_ms;
        return d;
    }

    void profile_start() {
        require("profile");
        check(e8qc_e8q_profile(idx_, 1, nullptr));
    }
    py::dict profile_stop() {
        require("profile");
        e8qc_profile p{};
        check(e8qc_e8q_profile(idx_, 0, &p));
        py::dict d;
        d["scan_launches"] = p.scan_launches;
        d["scan_ms"] = p.scan_ms;
        d["candidates"] = p.candidates;
        d["algo_bytes"] = p.algo_bytes;
        d["queries"] = p.queries;
        d["list_vectors"] = p.list_vectors;
        d["list_once"] = p.list_once;
        d["item_bytes"] = p.item_bytes;
        d["final_launches"] = p.final_launches;
        d["final_ms"] = p.final_ms;
        d["final_bytes"] = p.final_bytes;
        d["prep_ms"] = p.prep_ms;
        return d;
    }

    size_t dim() const { return dim_; }
    size_t nbits() const { return nbits_; }
    bool is_built() const { return built_; }
    size_t n() const { return built_ ? info().n : 0; }
    size_t num_clusters() const { return built_ ? info().nlist : 0; }
    size_t memory_bytes() const { return built_ ? info().memory_bytes : 0; }
    bool disable_prune() const { return built_ ? info().disable_prune != 0 : false; }
    int device() const { return device_; }

   private:
    void fresh() {
        if (idx_) e8qc_e8q_destroy(idx_);
        idx_ = nullptr;
        built_ = false;
        check(e8qc_e8q_create(device_, dim_, static_cast<int>(nbits_), seed_, &idx_));
    }
    void require(const char* what) const {
        if (!built_ || idx_ == nullptr)
            throw std::runtime_error(std::string("E8qIndex must be built or loaded before ") + what);
    }
    e8qc_info info() const {
        e8qc_info in{};
        check(e8qc_e8q_info(idx_, &in));
        return in;
    }
    py::dict stats_dict(const e8qc_stats& st, size_t nq, size_t nprobe) const {
        (void)nprobe;
        py::dict d;
        d["candidates"] = st.candidates;
        d["survivors"] = st.survivors;
        d["rotate_us"] = st.rotate_us / static_cast<double>(nq);
        d["route_us"] = st.route_us / static_cast<double>(nq);
        d["scan_us"] = st.scan_us / static_cast<double>(nq);
        d["refine_us"] = st.refine_us / static_cast<double>(nq);
        d["survivor_rate"] = st.candidates > 0 ? static_cast<double>(st.survivors) / st.candidates : 0.0;
        d["launches"] = st.launches;
        return d;
    }

    size_t dim_ = 0, nbits_ = 0;
    uint64_t seed_ = 0;
    int device_ = 0;
    bool built_ = false;
    e8qc_index* idx_ = nullptr;

   public:
    e8qc_index* handle(const char* what) const {
        require(what);
        return idx_;
    }

    // E8qIndex.save (e8q_bindings.cpp:258-263): a file the reference's load reads.
    void save(const std::string& path) const {
        require("save");
        py::gil_scoped_release nogil;
        check(e8qc_e8q_save(idx_, path.c_str()));
    }

    // E8qIndex.load (e8q_bindings.cpp:258-268): a reference-written index file.
    static std::unique_ptr<E8qIndex> load(const std::string& path, int device) {
        e8qc_index* h = nullptr;
        {
            py::gil_scoped_release nogil;
            check(e8qc_e8q_load(device, path.c_str(), &h));
        }
        e8qc_info in{};
        const int rc = e8qc_e8q_info(h, &in);
        if (rc != E8QC_OK) {
            e8qc_e8q_destroy(h);
            check(rc);
        }
        auto out = std::make_unique<E8qIndex>(static_cast<size_t>(in.dim), static_cast<size_t>(in.nbits), 0, device);
        out->idx_ = h;
        out->built_ = true;
        return out;
    }
};

// Me8qIndex (python_bindings/me8q_bindings.cpp:22-269 of the reference): same
// constructor, build / search / estimate arguments, properties and errors;
// `device` is this library's addition. save / load are not part of the
// device path.
class Me8qIndex {
   public:
    Me8qIndex(size_t dim, float avg_bits, uint64_t seed, int device)
        : dim_(dim), avg_bits_(avg_bits), seed_(seed), device_(device) {
        if (dim == 0) throw std::invalid_argument("dim must be positive");
        if (!(avg_bits > 0.0F)) throw std::invalid_argument("avg_bits must be positive");
    }
    ~Me8qIndex() {
        if (idx_) e8qc_me8q_destroy(idx_);
    }
    Me8qIndex(const Me8qIndex&) = delete;
    Me8qIndex& operator=(const Me8qIndex&) = delete;

    void build(py::handle data, py::handle centroids, py::handle cluster_ids, size_t /*num_threads*/,
               py::handle variance, bool drop_energy, float prune_alpha, const std::string& plan_spec,
               double extra_budget_bits) {
        auto x = ensure_nd<float>(data, "data", 2);
        auto c = ensure_nd<float>(centroids, "centroids", 2);
        auto ids = ensure_nd<uint32_t>(cluster_ids, "cluster_ids", 1);
        if (static_cast<size_t>(x.shape(1)) != dim_)
            throw std::invalid_argument("data dimension does not match index dim");
        if (static_cast<size_t>(c.shape(1)) != dim_)
            throw std::invalid_argument("centroid dimension does not match index dim");
        if (ids.shape(0) != x.shape(0))
            throw std::invalid_argument("cluster_ids length must match number of rows in data");
        py::array_t<float, py::array::c_style | py::array::forcecast> var;
        e8qc_me8q_build_opts o{};
        if (!variance.is_none()) {
            var = ensure_nd<float>(variance, "variance", 1);
            if (static_cast<size_t>(var.shape(0)) != dim_)
                throw std::invalid_argument("variance length must match dim");
            o.variance = var.data();
        }
        o.plan_spec = plan_spec.c_str();
        o.drop_energy = drop_energy ? 1 : 0;
        o.prune_alpha = prune_alpha;
        o.extra_budget_bits = extra_budget_bits;
        if (idx_) e8qc_me8q_destroy(idx_);
        idx_ = nullptr;
        built_ = false;
        check(e8qc_me8q_create(device_, dim_, avg_bits_, seed_, &idx_));
        {
            py::gil_scoped_release nogil;
            check(e8qc_me8q_build(idx_, x.data(), static_cast<size_t>(x.shape(0)), c.data(),
                                  static_cast<size_t>(c.shape(0)), ids.data(), &o, nullptr));
        }
        built_ = true;
    }

    // Device-resident build: raw CUDA pointers (e.g. torch tensor data_ptr());
    // variance 0 = computed from the data.
    void build_ptr(uintptr_t data, size_t n, uintptr_t centroids, size_t nlist, uintptr_t cluster_ids,
                   uintptr_t variance, bool drop_energy, const std::string& plan_spec, double extra_budget_bits,
                   uintptr_t stream) {
        e8qc_me8q_build_opts o{};
        o.variance = reinterpret_cast<const float*>(variance);
        o.plan_spec = plan_spec.c_str();
        o.drop_energy = drop_energy ? 1 : 0;
        o.extra_budget_bits = extra_budget_bits;
        if (idx_) e8qc_me8q_destroy(idx_);
        idx_ = nullptr;
        built_ = false;
        check(e8qc_me8q_create(device_, dim_, avg_bits_, seed_, &idx_));
        {
            py::gil_scoped_release nogil;
            check(e8qc_me8q_build(idx_, reinterpret_cast<const float*>(data), n,
                                  reinterpret_cast<const float*>(centroids), nlist,
                                  reinterpret_cast<const uint32_t*>(cluster_ids), &o, reinterpret_cast<void*>(stream)));
        }
        built_ = true;
    }

    // Device-resident search on raw CUDA pointers; returns the launch count.
    uint64_t search_ptr(uintptr_t queries, size_t nq, size_t k, size_t nprobe, uintptr_t out_ids, uintptr_t out_dists,
                        const std::string& mode, uintptr_t stream) {
        require("search");
        const int md = me8q_mode(mode);
        e8qc_stats st{};
        py::gil_scoped_release nogil;
        check(e8qc_me8q_search_mode(idx_, reinterpret_cast<const float*>(queries), nq, k, nprobe, md,
                                    reinterpret_cast<uint32_t*>(out_ids), reinterpret_cast<float*>(out_dists), &st,
                                    reinterpret_cast<void*>(stream)));
        return st.launches;
    }

    py::tuple search(py::handle queries, size_t k, size_t nprobe, size_t /*num_threads*/, bool return_stats,
                     const std::string& mode) {
        auto q = ensure_nd<float>(queries, "queries", 2);
        require("search");
        const int md = me8q_mode(mode);
        if (static_cast<size_t>(q.shape(1)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        if (k == 0) throw std::invalid_argument("k must be positive");
        if (k > E8QC_MAX_K) throw std::invalid_argument("k must be <= " + std::to_string(E8QC_MAX_K));
        if (nprobe == 0) throw std::invalid_argument("nprobe must be positive");
        const size_t nq = static_cast<size_t>(q.shape(0));
        py::array_t<uint32_t> ids({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k)});
        py::array_t<float> dists({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k)});
        uint32_t* ip = ids.mutable_data();
        float* dp = dists.mutable_data();
        std::fill(ip, ip + nq * k, std::numeric_limits<uint32_t>::max());
        std::fill(dp, dp + nq * k, std::numeric_limits<float>::infinity());
        e8qc_stats st{};
        {
            py::gil_scoped_release nogil;
            if (nq > 0)
                check(e8qc_me8q_search_mode(idx_, q.data(), nq, k, nprobe, md, ip, dp, return_stats ? &st : nullptr,
                                            nullptr));
        }
        if (!return_stats) return py::make_tuple(ids, dists);
        py::dict d;
        const double dn = nq > 0 ? static_cast<double>(nq) : 1.0;
        d["candidates"] = st.candidates;
        d["survivors"] = st.survivors;
        d["route_us"] = st.route_us / dn;
        d["scan_us"] = st.scan_us / dn;
        d["survivor_rate"] = st.candidates > 0 ? static_cast<double>(st.survivors) / st.candidates : 0.0;
        d["launches"] = st.launches;
        return py::make_tuple(ids, dists, d);
    }

    float estimate(py::handle query, uint32_t id) {
        require("estimate");
        auto q = ensure_nd<float>(query, "query", 1);
        if (static_cast<size_t>(q.shape(0)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        float out = 0.0f;
        const int rc = e8qc_me8q_estimate(idx_, q.data(), id, &out);
        if (rc == E8QC_ERANGE) throw py::index_error(e8qc_last_error());
        check(rc);
        return out;
    }

    // (ids, digits n x pd, branch n x pd/8, coef n x ncoded, h2 n x ncoded),
    // cluster-major.
    py::tuple export_codes() {
        require("export_codes");
        const e8qc_me8q_meta in = info();
        const auto n = static_cast<py::ssize_t>(in.n), pd = static_cast<py::ssize_t>(in.padded_dim),
                   nc = static_cast<py::ssize_t>(in.ncoded);
        py::array_t<uint32_t> ids(n);
        py::array_t<uint16_t> dg({n, pd});
        py::array_t<uint8_t> br({n, pd / 8});
        py::array_t<float> cf({n, nc}), h2({n, nc});
        check(e8qc_me8q_get_ids(idx_, ids.mutable_data()));
        check(e8qc_me8q_export_codes(idx_, dg.mutable_data(), br.mutable_data(), cf.mutable_data(), h2.mutable_data()));
        return py::make_tuple(ids, dg, br, cf, h2);
    }

    size_t dim() const { return dim_; }
    float avg_bits() const { return avg_bits_; }
    bool is_built() const { return built_; }
    size_t n() const { return idx_ ? info().n : 0; }
    size_t num_clusters() const { return idx_ ? info().nlist : 0; }
    double bits_per_dim() const { return idx_ ? info().bits_per_dim : 0.0; }
    size_t memory_bytes() const { return idx_ ? info().memory_bytes : 0; }
    int device() const { return device_; }
    std::vector<std::pair<size_t, int>> plan() const {
        std::vector<std::pair<size_t, int>> out;
        if (!idx_) return out;
        size_t cnt = 0;
        check(e8qc_me8q_plan(idx_, nullptr, nullptr, 0, &cnt));
        std::vector<size_t> lens(cnt);
        std::vector<int> bits(cnt);
        check(e8qc_me8q_plan(idx_, lens.data(), bits.data(), cnt, &cnt));
        for (size_t i = 0; i < cnt; ++i) out.emplace_back(lens[i], bits[i]);
        return out;
    }

    // Serving form: per-query k and nprobe; rows padded to k_max.
    py::tuple search_ragged(py::handle queries, py::handle k, py::handle nprobe, size_t k_max,
                            const std::string& mode) {
        const int md = me8q_mode(mode);
        auto q = ensure_nd<float>(queries, "queries", 2);
        auto ka = ensure_nd<uint32_t>(k, "k", 1);
        auto na = ensure_nd<uint32_t>(nprobe, "nprobe", 1);
        require("search");
        if (static_cast<size_t>(q.shape(1)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        const size_t nq = static_cast<size_t>(q.shape(0));
        if (static_cast<size_t>(ka.shape(0)) != nq || static_cast<size_t>(na.shape(0)) != nq)
            throw std::invalid_argument("k and nprobe must have one entry per query");
        py::array_t<uint32_t> ids({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k_max)});
        py::array_t<float> dists({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k_max)});
        {
            py::gil_scoped_release nogil;
            if (nq > 0)
                check(e8qc_me8q_search_ragged(idx_, q.data(), nq, ka.data(), na.data(), k_max, md,
                                              ids.mutable_data(), dists.mutable_data(), nullptr));
        }
        return py::make_tuple(ids, dists);
    }

    e8qc_me8q* handle(const char* what) const {
        require(what);
        return idx_;
    }

    // Me8qIndex.save (me8q_bindings.cpp:220-225): a file the reference loads.
    void save(const std::string& path) {
        require("save");
        py::gil_scoped_release nogil;
        check(e8qc_me8q_save(idx_, path.c_str()));
    }

    // Me8qIndex.load (me8q_bindings.cpp:227-235): a reference-written index file.
    static std::unique_ptr<Me8qIndex> load(const std::string& path, int device) {
        e8qc_me8q* h = nullptr;
        {
            py::gil_scoped_release nogil;
            check(e8qc_me8q_load(device, path.c_str(), &h));
        }
        e8qc_me8q_meta in{};
        const int rc = e8qc_me8q_info(h, &in);
        if (rc != E8QC_OK) {
            e8qc_me8q_destroy(h);
            check(rc);
        }
        // as the reference's load: avg_bits reports the stored rate (bits_per_dim)
        const float avg = in.bits_per_dim > 0.0 ? static_cast<float>(in.bits_per_dim) : in.avg_bits;
        auto out = std::make_unique<Me8qIndex>(static_cast<size_t>(in.dim), avg, 0, device);
        out->idx_ = h;
        out->built_ = true;
        return out;
    }

   private:
    void require(const char* what) const {
        if (!built_ || idx_ == nullptr)
            throw std::runtime_error(std::string("Me8qIndex must be built or loaded before ") + what);
    }
    e8qc_me8q_meta info() const {
        e8qc_me8q_meta in{};
        check(e8qc_me8q_info(idx_, &in));
        return in;
    }
    size_t dim_ = 0;
    float avg_bits_ = 4.0F;
    uint64_t seed_ = 0;
    int device_ = 0;
    bool built_ = false;
    e8qc_me8q* idx_ = nullptr;
};

// Captured search plan (see e8qc_plan_* in e8qc.h): one CUDA graph per
// batch size bucket. Holds a reference to the Python index.
class Plan {
   public:
    Plan(py::object index, const std::string& mode, size_t max_queries, size_t k_max, size_t nprobe_max,
         bool autotune)
        : index_(index), k_max_(k_max) {
        if (py::isinstance<Me8qIndex>(index)) {
            Me8qIndex& mx = index.cast<Me8qIndex&>();
            dim_ = mx.dim();
            const int md = me8q_mode(mode.empty() ? std::string("batched") : mode);
            e8qc_me8q* h = mx.handle("plan");
            py::gil_scoped_release nogil;
            check(e8qc_plan_create_me8q(h, md, max_queries, k_max, nprobe_max, autotune ? 1 : 0, &plan_));
            return;
        }
        E8qIndex& ix = index.cast<E8qIndex&>();
        dim_ = ix.dim();
        const int md = mode_of(mode.empty() ? std::string("precision") : mode);
        if (md == E8QC_MODE_PLAIN) throw std::invalid_argument("plans run 'batched' or 'precision'");
        e8qc_index* h = ix.handle("plan");
        py::gil_scoped_release nogil;
        check(e8qc_plan_create(h, md, max_queries, k_max, nprobe_max, autotune ? 1 : 0, &plan_));
    }
    ~Plan() {
        if (plan_) e8qc_plan_destroy(plan_);
    }
    py::tuple run(py::handle queries, py::handle k, py::handle nprobe) {
        auto q = ensure_nd<float>(queries, "queries", 2);
        if (static_cast<size_t>(q.shape(1)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        const size_t nq = static_cast<size_t>(q.shape(0));
        std::vector<uint32_t> kv(nq), nv(nq);
        auto fill = [&](py::handle h, std::vector<uint32_t>& v, const char* name) {
            if (py::isinstance<py::int_>(h)) {
                std::fill(v.begin(), v.end(), h.cast<uint32_t>());
            } else {
                auto a = ensure_nd<uint32_t>(h, name, 1);
                if (static_cast<size_t>(a.shape(0)) != nq)
                    throw std::invalid_argument(std::string(name) + " must have one entry per query");
                std::copy(a.data(), a.data() + nq, v.begin());
            }
        };
        fill(k, kv, "k");
        fill(nprobe, nv, "nprobe");
        py::array_t<uint32_t> ids({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k_max_)});
        py::array_t<float> dists({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k_max_)});
        if (nq > 0) {
            py::gil_scoped_release nogil;
            check(e8qc_plan_run(plan_, q.data(), nq, kv.data(), nv.data(), ids.mutable_data(), dists.mutable_data(),
                                nullptr));
        }
        return py::make_tuple(ids, dists);
    }

   private:
    py::object index_;
    size_t dim_ = 0, k_max_ = 0;
    e8qc_plan* plan_ = nullptr;
};

// Serving loop over one index (an addition of this library; see
// e8qc_server_* in e8qc.h). Holds a reference to the Python index so it
// outlives the server.
class Server {
   public:
    Server(py::object index, const std::string& mode, size_t max_batch, size_t max_k, size_t max_nprobe,
           size_t memory_budget, int slots, int request_timeout_ms)
        : index_(index) {
        e8qc_server_config c{};
        c.request_timeout_ms = request_timeout_ms;
        c.max_batch_queries = max_batch;
        c.max_k = max_k;
        c.max_nprobe = max_nprobe;
        c.memory_budget = memory_budget;
        c.slots = slots;
        if (py::isinstance<Me8qIndex>(index)) {
            Me8qIndex& mx = index.cast<Me8qIndex&>();
            dim_ = mx.dim();
            c.mode = me8q_mode(mode.empty() ? std::string("batched") : mode);
            e8qc_me8q* h = mx.handle("serve");
            py::gil_scoped_release nogil;
            check(e8qc_server_start_me8q(h, &c, &srv_));
            return;
        }
        E8qIndex& ix = index.cast<E8qIndex&>();
        dim_ = ix.dim();
        c.mode = mode_of(mode.empty() ? std::string("precision") : mode);
        if (c.mode == E8QC_MODE_PLAIN) throw std::invalid_argument("the server runs 'batched' or 'precision'");
        e8qc_index* h = ix.handle("serve");
        py::gil_scoped_release nogil;
        check(e8qc_server_start(h, &c, &srv_));
    }
    ~Server() {
        try {
            stop();
        } catch (...) {
        }
    }
    uint64_t submit(py::handle queries, size_t k, size_t nprobe) {
        if (!srv_) throw std::runtime_error("server is stopped");
        auto q = ensure_nd<float>(queries, "queries", 2);
        if (static_cast<size_t>(q.shape(1)) != dim_)
            throw std::invalid_argument("query dimension does not match index dim");
        const size_t nq = static_cast<size_t>(q.shape(0));
        uint64_t id = 0;
        {
            py::gil_scoped_release nogil;
            check(e8qc_server_submit(srv_, q.data(), nq, k, nprobe, &id));
        }
        shapes_[id] = {nq, k};
        return id;
    }
    py::object result(uint64_t id, int timeout_ms) {
        if (!srv_) throw std::runtime_error("server is stopped");
        auto it = shapes_.find(id);
        if (it == shapes_.end()) throw py::index_error("unknown or already collected request id");
        const size_t nq = it->second.first, k = it->second.second;
        py::array_t<uint32_t> ids({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k)});
        py::array_t<float> dists({static_cast<py::ssize_t>(nq), static_cast<py::ssize_t>(k)});
        int done = 0, rc = 0;
        {
            py::gil_scoped_release nogil;
            rc = e8qc_server_poll(srv_, id, timeout_ms, ids.mutable_data(), dists.mutable_data(), &done);
        }
        if (done) shapes_.erase(id);
        check(rc);
        if (!done) return py::none();
        return py::make_tuple(ids, dists);
    }
    // Cancel a request (e8qc_server_cancel): its result() then raises unless
    // it had already completed.
    void cancel(uint64_t id) {
        if (!srv_) throw std::runtime_error("server is stopped");
        const int rc = e8qc_server_cancel(srv_, id);
        if (rc == E8QC_ERANGE) throw py::index_error(e8qc_last_error());
        check(rc);
    }
    py::dict stats(bool reset) {
        if (!srv_) throw std::runtime_error("server is stopped");
        e8qc_server_stats st{};
        check(e8qc_server_get_stats(srv_, reset ? 1 : 0, &st));
        py::dict d;
        d["submitted"] = st.submitted;
        d["rejected"] = st.rejected;
        d["completed"] = st.completed;
        d["failed"] = st.failed;
        d["queries_completed"] = st.queries_completed;
        d["batches"] = st.batches;
        d["p50_ms"] = st.p50_ms;
        d["p99_ms"] = st.p99_ms;
        d["mean_ms"] = st.mean_ms;
        d["max_ms"] = st.max_ms;
        d["qps"] = st.qps;
        d["mean_batch_queries"] = st.mean_batch_queries;
        d["peak_batch_bytes"] = st.peak_batch_bytes;
        d["canceled"] = st.canceled;
        d["expired"] = st.expired;
        return d;
    }
    void stop() {
        if (!srv_) return;
        e8qc_server* s = srv_;
        srv_ = nullptr;
        int rc = 0;
        {
            py::gil_scoped_release nogil;
            rc = e8qc_server_stop(s);
        }
        check(rc);
    }

   private:
    py::object index_;
    size_t dim_ = 0;
    e8qc_server* srv_ = nullptr;
    std::unordered_map<uint64_t, std::pair<size_t, size_t>> shapes_;
};

}  // namespace e8qb200

PYBIND11_MODULE(_e8qlib, m) {
    using e8qb200::E8qIndex;
    m.doc() = "E8Q IVF search on B200 (sm_100a): the e8qlib Python API over libe8qcuda.so";
    m.def("version", [] { return e8qc_version(); });
    // Fault injection (no reference counterpart): the next `count` checked
    // host allocations fail (index creation, server request intake).
    m.def("debug_fail_host_allocs", [](int count) { e8qb200::check(e8qc_debug_fail_host_allocs(count)); }, py::arg("count"));
    m.def("branch_levels", [](int bits, int branch) {
        py::array_t<double> out(static_cast<py::ssize_t>(1) << std::max(1, std::min(bits, 13)));
        e8qb200::check(e8qc_branch_levels(bits, branch, out.mutable_data()));
        return out;
    }, py::arg("bits"), py::arg("branch"));
    m.def("fixed_scale", [](int bits) {
        double s = 0.0;
        e8qb200::check(e8qc_fixed_scale(bits, &s));
        return s;
    }, py::arg("bits"));
    m.def("encode", [](py::handle unit, int bits, int device) {
        auto u = e8qb200::ensure_nd<float>(unit, "unit", 2);
        const size_t n = static_cast<size_t>(u.shape(0)), pd = static_cast<size_t>(u.shape(1));
        py::array_t<uint16_t> dg({static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(pd / 8), py::ssize_t(8)});
        py::array_t<uint8_t> br({static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(pd / 8)});
        {
            py::gil_scoped_release nogil;
            e8qb200::check(e8qc_encode(device, bits, u.data(), n, pd, dg.mutable_data(), br.mutable_data(), nullptr));
        }
        return py::make_tuple(dg, br);
    }, py::arg("unit"), py::arg("bits"), py::arg("device") = 0);
    m.def("rotate", [](py::handle x, size_t dim, uint64_t seed, int device) {
        auto a = e8qb200::ensure_nd<float>(x, "x", 2);
        if (static_cast<size_t>(a.shape(1)) != dim) throw std::invalid_argument("x dimension does not match dim");
        const size_t n = static_cast<size_t>(a.shape(0)), pd = (dim + 63) / 64 * 64;
        py::array_t<float> out({static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(pd)});
        {
            py::gil_scoped_release nogil;
            e8qb200::check(e8qc_rotate(device, dim, seed, a.data(), n, out.mutable_data(), nullptr));
        }
        return out;
    }, py::arg("x"), py::arg("dim"), py::arg("seed"), py::arg("device") = 0);

    m.def("tc_i8_gemm", [](py::handle a, py::handle b, int reps, int grid, int device) {
        auto A = e8qb200::ensure_nd<int8_t>(a, "A", 2);
        auto B = e8qb200::ensure_nd<int8_t>(b, "B", 2);
        if (A.shape(0) != 128 || A.shape(1) != B.shape(1)) throw std::invalid_argument("A must be 128 x k, B n x k");
        const int n = static_cast<int>(B.shape(0)), k = static_cast<int>(A.shape(1));
        py::array_t<int32_t> C({py::ssize_t(128), static_cast<py::ssize_t>(n)});
        float ms = 0.0f;
        {
            py::gil_scoped_release nogil;
            e8qb200::check(e8qc_tc_i8_gemm(device, A.data(), B.data(), n, k, reps, grid, C.mutable_data(), &ms));
        }
        return py::make_tuple(C, ms);
    }, py::arg("A"), py::arg("B"), py::arg("reps") = 1, py::arg("grid") = 1, py::arg("device") = 0);

    py::class_<e8qb200::Plan>(m, "Plan")
        .def(py::init<py::object, const std::string&, size_t, size_t, size_t, bool>(), py::arg("index"),
             py::arg("mode") = "", py::arg("max_queries") = 4096, py::arg("k_max") = 10,
             py::arg("nprobe_max") = 64, py::arg("autotune") = true)
        .def("run", &e8qb200::Plan::run, py::arg("queries"), py::arg("k"), py::arg("nprobe"));

    py::class_<e8qb200::Server>(m, "Server")
        .def(py::init<py::object, const std::string&, size_t, size_t, size_t, size_t, int, int>(),
             py::arg("index"), py::arg("mode") = "", py::arg("max_batch") = 4096, py::arg("max_k") = 128,
             py::arg("max_nprobe") = 0, py::arg("memory_budget") = 0, py::arg("slots") = 2,
             py::arg("request_timeout_ms") = 0)
        .def("cancel", &e8qb200::Server::cancel, py::arg("request_id"))
        .def("submit", &e8qb200::Server::submit, py::arg("queries"), py::arg("k"), py::arg("nprobe"))
        .def("result", &e8qb200::Server::result, py::arg("request_id"), py::arg("timeout_ms") = -1)
        .def("stats", &e8qb200::Server::stats, py::arg("reset") = false)
        .def("stop", &e8qb200::Server::stop)
        .def("__enter__", [](py::object self) { return self; })
        .def("__exit__", [](e8qb200::Server& s, py::args) { s.stop(); });

    py::class_<e8qb200::Me8qIndex>(m, "Me8qIndex")
        .def(py::init<size_t, float, uint64_t, int>(), py::arg("dim"), py::arg("avg_bits") = 4.0F,
             py::arg("seed") = 0, py::arg("device") = 0)
        .def("build", &e8qb200::Me8qIndex::build, py::arg("data"), py::arg("centroids"), py::arg("cluster_ids"),
             py::arg("num_threads") = 1, py::arg("variance") = py::none(), py::arg("drop_energy") = true,
             py::arg("prune_alpha") = 0.0F, py::arg("plan_spec") = "", py::arg("extra_budget_bits") = 0.0)
        .def("search", &e8qb200::Me8qIndex::search, py::arg("queries"), py::arg("k"), py::arg("nprobe"),
             py::arg("num_threads") = 1, py::arg("return_stats") = false, py::arg("mode") = "pruned")
        .def("estimate", &e8qb200::Me8qIndex::estimate, py::arg("query"), py::arg("id"))
        .def_static("load", &e8qb200::Me8qIndex::load, py::arg("path"), py::arg("device") = 0)
        .def("save", &e8qb200::Me8qIndex::save, py::arg("path"))
        .def("export_codes", &e8qb200::Me8qIndex::export_codes)
        .def("search_ragged", &e8qb200::Me8qIndex::search_ragged, py::arg("queries"), py::arg("k"),
             py::arg("nprobe"), py::arg("k_max"), py::arg("mode") = "batched")
        .def("build_ptr", &e8qb200::Me8qIndex::build_ptr, py::arg("data"), py::arg("n"), py::arg("centroids"),
             py::arg("nlist"), py::arg("cluster_ids"), py::arg("variance") = 0, py::arg("drop_energy") = true,
             py::arg("plan_spec") = "", py::arg("extra_budget_bits") = 0.0, py::arg("stream") = 0)
        .def("search_ptr", &e8qb200::Me8qIndex::search_ptr, py::arg("queries"), py::arg("nq"), py::arg("k"),
             py::arg("nprobe"), py::arg("out_ids"), py::arg("out_dists"), py::arg("mode") = "batched",
             py::arg("stream") = 0)
        .def_property_readonly("dim", &e8qb200::Me8qIndex::dim)
        .def_property_readonly("avg_bits", &e8qb200::Me8qIndex::avg_bits)
        .def_property_readonly("is_built", &e8qb200::Me8qIndex::is_built)
        .def_property_readonly("n", &e8qb200::Me8qIndex::n)
        .def_property_readonly("num_clusters", &e8qb200::Me8qIndex::num_clusters)
        .def_property_readonly("bits_per_dim", &e8qb200::Me8qIndex::bits_per_dim)
        .def_property_readonly("memory_bytes", &e8qb200::Me8qIndex::memory_bytes)
        .def_property_readonly("plan", &e8qb200::Me8qIndex::plan)
        .def_property_readonly("device", &e8qb200::Me8qIndex::device);

    py::class_<E8qIndex>(m, "E8qIndex")
        .def(py::init<size_t, size_t, uint64_t, int>(), py::arg("dim"), py::arg("nbits"),
             py::arg("seed") = 0, py::arg("device") = 0)
        .def("build", &E8qIndex::build, py::arg("data"), py::arg("centroids"), py::arg("cluster_ids"),
             py::arg("num_threads") = 1, py::arg("prune_alpha") = 0.0F)
        .def("build_ptr", &E8qIndex::build_ptr, py::arg("data"), py::arg("n"), py::arg("centroids"),
             py::arg("nlist"), py::arg("cluster_ids"), py::arg("prune_alpha") = 0.0F,
             py::arg("stream") = 0)
        .def("search", &E8qIndex::search, py::arg("queries"), py::arg("k"), py::arg("nprobe"),
             py::arg("num_threads") = 1, py::arg("return_stats") = false, py::arg("mode") = "auto")
        .def("pruned_thresholds", &E8qIndex::pruned_thresholds, py::arg("nq"))
        .def("search_ptr", &E8qIndex::search_ptr, py::arg("queries"), py::arg("nq"), py::arg("k"),
             py::arg("nprobe"), py::arg("out_ids"), py::arg("out_dists"), py::arg("mode") = "auto",
             py::arg("stream") = 0)
        .def("search_ragged", &E8qIndex::search_ragged, py::arg("queries"), py::arg("k"),
             py::arg("nprobe"), py::arg("k_max"), py::arg("mode") = "batched")
        .def("estimate", &E8qIndex::estimate, py::arg("query"), py::arg("id"))
        .def_static("load", &E8qIndex::load, py::arg("path"), py::arg("device") = 0)
        .def("save", &E8qIndex::save, py::arg("path"))
        .def("autotune", &E8qIndex::autotune, py::arg("mode"), py::arg("nq"), py::arg("k"), py::arg("nprobe"))
        .def("set_disable_prune", &E8qIndex::set_disable_prune, py::arg("on"))
        .def("probe_bound_w", &E8qIndex::probe_bound_w, py::arg("queries"), py::arg("base"), py::arg("qidx"),
             py::arg("ids"), py::arg("num_threads") = 1)
        .def("debug_inject_wait_timeout", &E8qIndex::debug_inject_wait_timeout, py::arg("searches"),
             py::arg("wait_ms") = 50)
        .def("set_prune_alpha", &E8qIndex::set_prune_alpha, py::arg("alpha"))
        .def("export_codes", &E8qIndex::export_codes)
        .def("profile_start", &E8qIndex::profile_start)
        .def("profile_stop", &E8qIndex::profile_stop)
        .def_property_readonly("dim", &E8qIndex::dim)
        .def_property_readonly("nbits", &E8qIndex::nbits)
        .def_property_readonly("is_built", &E8qIndex::is_built)
        .def_property_readonly("n", &E8qIndex::n)
        .def_property_readonly("num_clusters", &E8qIndex::num_clusters)
        .def_property_readonly("memory_bytes", &E8qIndex::memory_bytes)
        .def_property_readonly("disable_prune", &E8qIndex::disable_prune)
        .def_property_readonly("device", &E8qIndex::device);
}
