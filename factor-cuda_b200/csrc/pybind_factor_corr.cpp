// pybind_factor_corr.cpp -- drop-in `factor_corr_pybind` module over the C ABI.
//
// Same surface as the reference binding (src/factor_corr_pybind.cpp:38-108):
// factor_corr_f64(F3, mask=None) -> (F,F) f64, F3 a (T,N,F) numeric panel
// (any real dtype is accepted and widened, as the reference's forcecast does;
// f32 is passed at its own width), mask None or (T,N) castable to uint8.
// Shape/F caps raise ValueError; any other non-zero status raises
// RuntimeError, as in the reference binding.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/fcb200.h"

namespace py = pybind11;

using ArrF32 = py::array_t<float, py::array::c_style>;
using ArrD = py::array_t<double, py::array::c_style | py::array::forcecast>;
using ArrU8 = py::array_t<uint8_t, py::array::c_style | py::array::forcecast>;

static py::array_t<double> factor_corr_f64(py::object F3, py::object mask) {
  py::array panel;
  int dtype;
  if (py::isinstance<py::array>(F3) &&
      py::reinterpret_borrow<py::array>(F3).dtype() == py::dtype::of<float>()) {
    panel = py::cast<ArrF32>(F3);
    dtype = FCB_DTYPE_F32;
  } else {
    panel = py::cast<ArrD>(F3);
    dtype = FCB_DTYPE_F64;
  }
  if (panel.ndim() != 3) throw std::invalid_argument("F3 must be 3-D (T,N,F)");
  const py::ssize_t T = panel.shape(0), N = panel.shape(1), F = panel.shape(2);
  if (T < 1 || N < 1 || F < 1) throw std::invalid_argument("F3 shape must be (T,N,F) with T,N,F >= 1");
  if (static_cast<int64_t>(T) * N > INT32_MAX) throw std::invalid_argument("T*N exceeds INT32_MAX (implementation cap)");
  if (F > 128) throw std::invalid_argument("F > 128 (factor pair grid cap)");
  ArrU8 mh;
  const uint8_t* mp = nullptr;
  if (!mask.is_none()) {
    mh = mask.cast<ArrU8>();
    if (mh.ndim() != 2 || mh.shape(0) != T || mh.shape(1) != N)
      throw std::invalid_argument("mask shape must be (T,N) matching F3");
    mp = mh.data();
  }
  py::array_t<double> out({F, F});
  double* op = out.mutable_data();
  const void* xp = panel.data();
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = fcb_factor_corr(xp, dtype, mp, static_cast<int>(T), static_cast<int>(N), static_cast<int>(F), op, nullptr);
  }
  if (rc != 0)
    throw std::runtime_error("factor_corr_gpu failed with error code " + std::to_string(rc) + " (" +
                             fcb_status_string(rc) + ")");
  return out;
}

PYBIND11_MODULE(factor_corr_pybind, m) {
  m.doc() =
      "B200 (sm_100a) drop-in for factor-cuda's factor_corr_pybind module.\n"
      "  factor_corr_f64(F3, mask=None) -> (F,F) float64\n"
      "Compute runs in libfcb200.so (C ABI, include/fcb200.h).";
  m.def("factor_corr_f64", &factor_corr_f64, py::arg("F3"), py::arg("mask") = py::none(),
        "(F,F) pooled pairwise-complete factor correlation of a (T,N,F) panel.");
}
