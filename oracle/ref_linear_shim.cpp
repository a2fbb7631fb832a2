// Test-only shim around the reference linear scan (competitors/linear/src/linear_index.cpp).
//
// ORACLE INFRASTRUCTURE: this file is compiled only into oracle/_ref/ and is imported only by
// tests/, the smoke check and bench.py's CPU-baseline leg. It never ships in the product path.
//
// The reference translation unit is #included unchanged from where it lies (the include path
// points at the reference source tree). Its PYBIND11_MODULE block is turned into a plain
// registration function so this module can register the reference class under its own name
// ("LinearIndex") and add one probe: the reference's inline compute_l2_distance
// (competitors/linear/src/simd.h:32-115), so tests can compare summation order bit-for-bit.
#include <pybind11/pybind11.h>
#include <pybind11/numpy.h>
#include <pybind11/stl.h>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <thread>
#include <vector>

#pragma push_macro("PYBIND11_MODULE")
#undef PYBIND11_MODULE
#define PYBIND11_MODULE(name, variable) static void annvedi_ref_register_##name(pybind11::module_ &variable)
#include "linear_index.cpp"
#pragma pop_macro("PYBIND11_MODULE")

namespace py = pybind11;

PYBIND11_MODULE(ref_linear_shim, m) {
    annvedi_ref_register_linear_ann_cpp(m);
    m.def("l2_distance",
          [](py::array_t<float, py::array::c_style | py::array::forcecast> a,
             py::array_t<float, py::array::c_style | py::array::forcecast> b, float threshold) {
              if (a.size() != b.size()) throw std::runtime_error("size mismatch");
              return compute_l2_distance(a.data(), b.data(), (size_t)a.size(), threshold);
          },
          py::arg("a"), py::arg("b"), py::arg("threshold") = std::numeric_limits<float>::max());
#if defined(HAS_AVX512)
    m.attr("simd") = "avx512";
#elif defined(HAS_AVX)
    m.attr("simd") = "avx2";
#else
    m.attr("simd") = "scalar";
#endif
}
