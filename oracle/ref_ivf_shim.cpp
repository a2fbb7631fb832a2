// Test-only shim around the reference per-dimension SQ8 IVF-LSH index
// (competitors/ivf_lsh/src/lsh_index_optimized.cpp).
//
// ORACLE INFRASTRUCTURE: compiled only into oracle/_ref/; imported only by tests/, the smoke
// check and bench.py's CPU-baseline leg. Never part of the product path.
//
// The reference translation unit is #included unchanged from where it lies. Two things are
// added around it, both test plumbing:
//   * state export/import, so a GPU index and the reference answer queries over the SAME
//     centroids, codes, scales and inverted lists (the reference's k-means depends on the host
//     thread count, lsh_index_optimized.cpp:61-73,594-601, so fit() itself is not portable);
//   * set_num_threads, which replaces the reference's ThreadPool (sized from
//     hardware_concurrency() at lsh_index_optimized.cpp:140) so the SQ8 pass's per-chunk
//     64-entry heaps (:86-122, :465-469) are reproducible on any host.
//   * set_fit_threads, which pins the thread count fit() reads from hardware_concurrency()
//     (:140): its k-means sums per ThreadPool chunk (:61-73, :594-601), so a fit is reproducible
//     only with the count fixed. The reference asks std::thread for it on one line (:140); within
//     the reference include the token `thread` names a stand-in whose hardware_concurrency()
//     returns the pinned count (0 = the real one). No other `thread` token appears in code there.
// Member access uses a preprocessor override of `private`, confined to the reference include.
#include <pybind11/pybind11.h>
#include <pybind11/numpy.h>
#include <pybind11/stl.h>
#include <pthread.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <limits>
#include <memory>
#include <numeric>
#include <random>
#include <stdexcept>
#include <thread>
#include <unordered_map>
#include <vector>
#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace annvedi_shim {
static int g_fit_threads = 0;
struct pinned_thread {
    static unsigned hardware_concurrency() noexcept {
        return g_fit_threads > 0 ? (unsigned)g_fit_threads : std::thread::hardware_concurrency();
    }
};
}  // namespace annvedi_shim
namespace std {
using annvedi_pinned_thread = ::annvedi_shim::pinned_thread;
}

#pragma push_macro("PYBIND11_MODULE")
#undef PYBIND11_MODULE
#define PYBIND11_MODULE(name, variable) static void annvedi_ref_register_##name(pybind11::module_ &variable)
#define private public
#define thread annvedi_pinned_thread
#include "lsh_index_optimized.cpp"
#undef thread
#undef private
#pragma pop_macro("PYBIND11_MODULE")

namespace py = pybind11;
using f32arr = py::array_t<float, py::array::c_style | py::array::forcecast>;
using u8arr = py::array_t<uint8_t, py::array::c_style | py::array::forcecast>;
using i32arr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;
using i64arr = py::array_t<int64_t, py::array::c_style | py::array::forcecast>;

static py::dict export_state(const IVFLSHIndex &ix) {
    py::dict d;
    const int N = ix.npts_, D = ix.dim_, C = ix.n_clusters_;
    const int T = ix.n_tables_, B = ix.n_bits_;
    d["npts"] = N;
    d["dim"] = D;
    d["n_clusters"] = C;
    d["n_tables"] = T;
    d["n_bits"] = B;
    d["num_threads"] = ix.pool_ ? ix.pool_->get_num_threads() : 0;
    d["centroids"] = f32arr({C, D}, ix.centroids_.data());
    d["original_data"] = f32arr({N, D}, ix.original_data_.data());
    d["quantized_data"] = u8arr({N, D}, ix.quantized_data_.data());
    d["scale"] = f32arr({D}, ix.scale_.data());
    d["offset"] = f32arr({D}, ix.offset_.data());
    d["mean"] = f32arr({D}, ix.mean_.data());
    d["reordered_to_original"] = i32arr({N}, ix.reordered_to_original_.data());
    std::vector<float> proj((size_t)T * B * D);
    for (int i = 0; i < T * B; ++i)
        std::copy(ix.projections_[i].begin(), ix.projections_[i].end(), proj.begin() + (size_t)i * D);
    d["projections"] = f32arr({T * B, D}, proj.data());
    const int nb = 1 << B;
    std::vector<int64_t> off((size_t)T * C * nb + 1, 0);
    std::vector<int32_t> ids;
    size_t pos = 0;
    for (int t = 0; t < T; ++t)
        for (int c = 0; c < C; ++c)
            for (int s = 0; s < nb; ++s) {
                const auto &b = ix.tables_[t][c][s];
                off[pos++] = (int64_t)ids.size();
                ids.insert(ids.end(), b.begin(), b.end());
            }
    off[pos] = (int64_t)ids.size();
    d["table_offsets"] = i64arr({(py::ssize_t)off.size()}, off.data());
    d["table_ids"] = i32arr({(py::ssize_t)ids.size()}, ids.data());
    return d;
}

static void import_state(IVFLSHIndex &ix, py::dict d, int num_threads) {
    const int N = d["npts"].cast<int>(), D = d["dim"].cast<int>(), C = d["n_clusters"].cast<int>();
    const int T = d["n_tables"].cast<int>(), B = d["n_bits"].cast<int>();
    ix.npts_ = N;
    ix.dim_ = D;
    ix.n_clusters_ = C;
    ix.n_tables_ = T;
    ix.n_bits_ = B;
    auto cen = d["centroids"].cast<f32arr>();
    auto orig = d["original_data"].cast<f32arr>();
    auto q8 = d["quantized_data"].cast<u8arr>();
    auto sc = d["scale"].cast<f32arr>();
    auto of = d["offset"].cast<f32arr>();
    auto mn = d["mean"].cast<f32arr>();
    auto r2o = d["reordered_to_original"].cast<i32arr>();
    auto proj = d["projections"].cast<f32arr>();
    auto toff = d["table_offsets"].cast<i64arr>();
    auto tids = d["table_ids"].cast<i32arr>();
    if (cen.size() != (py::ssize_t)C * D || orig.size() != (py::ssize_t)N * D || q8.size() != (py::ssize_t)N * D ||
        sc.size() != D || of.size() != D || mn.size() != D || r2o.size() != N ||
        proj.size() != (py::ssize_t)T * B * D || toff.size() != (py::ssize_t)T * C * (1 << B) + 1)
        throw std::runtime_error("import_state: inconsistent array sizes");
    ix.centroids_.assign(cen.data(), cen.data() + cen.size());
    ix.original_data_.assign(orig.data(), orig.data() + orig.size());
    ix.data_.clear();
    ix.quantized_data_.assign(q8.data(), q8.data() + q8.size());
    ix.scale_.assign(sc.data(), sc.data() + D);
    ix.offset_.assign(of.data(), of.data() + D);
    ix.mean_.assign(mn.data(), mn.data() + D);
    ix.reordered_to_original_.assign(r2o.data(), r2o.data() + N);
    ix.projections_.assign((size_t)T * B, std::vector<float>(D));
    for (int i = 0; i < T * B; ++i)
        std::copy(proj.data() + (size_t)i * D, proj.data() + (size_t)(i + 1) * D, ix.projections_[i].begin());
    const int nb = 1 << B;
    ix.tables_.assign(T, std::vector<std::vector<std::vector<int32_t>>>(C, std::vector<std::vector<int32_t>>(nb)));
    size_t pos = 0;
    for (int t = 0; t < T; ++t)
        for (int c = 0; c < C; ++c)
            for (int s = 0; s < nb; ++s, ++pos)
                ix.tables_[t][c][s].assign(tids.data() + toff.data()[pos], tids.data() + toff.data()[pos + 1]);
    ix.visited_query_ids_.assign(N, 0);
    ix.current_query_id_ = 0;
    ix.pool_ = std::make_unique<ThreadPool>(num_threads > 0 ? num_threads : 1);
    ix.n_distances_ = 0;
    ix.reset_profile_results();
}

PYBIND11_MODULE(ref_ivf_shim, m) {
    annvedi_ref_register_ivf_lsh_cpp(m);
    m.def("export_state", &export_state);
    m.def("import_state", &import_state, py::arg("index"), py::arg("state"), py::arg("num_threads"));
    m.def("set_num_threads", [](IVFLSHIndex &ix, int t) { ix.pool_ = std::make_unique<ThreadPool>(t > 0 ? t : 1); });
    m.def("set_fit_threads", [](int t) { annvedi_shim::g_fit_threads = t > 0 ? t : 0; });
    m.def("get_num_threads", [](const IVFLSHIndex &ix) { return ix.pool_ ? ix.pool_->get_num_threads() : 0; });
    m.def("l2_distance",
          [](f32arr a, f32arr b, float threshold) {
              if (a.size() != b.size()) throw std::runtime_error("size mismatch");
              return compute_l2_distance(a.data(), b.data(), (size_t)a.size(), threshold);
          },
          py::arg("a"), py::arg("b"), py::arg("threshold") = std::numeric_limits<float>::max());
    m.def("l2_distance_sq8",
          [](u8arr code, f32arr q_shifted, f32arr scale, float threshold) {
              if (code.size() != q_shifted.size() || code.size() != scale.size())
                  throw std::runtime_error("size mismatch");
              return compute_l2_distance_quantized(code.data(), q_shifted.data(), (size_t)code.size(),
                                                   scale.data(), threshold);
          },
          py::arg("code"), py::arg("q_shifted"), py::arg("scale"),
          py::arg("threshold") = std::numeric_limits<float>::max());
#if defined(HAS_AVX512)
    m.attr("simd") = "avx512";
#elif defined(HAS_AVX)
    m.attr("simd") = "avx2";
#else
    m.attr("simd") = "scalar";
#endif
}
