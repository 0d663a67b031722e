// pybind_factor_cuda.cpp -- drop-in `factor_cuda_pybind` module over the C ABI.
//
// Same Python-level surface as the reference binding
// (src/factor_cuda_pybind.cpp:439-536): cs_rank_f32, rolling_ic_f64,
// stock_corr_f64, parameter_scan_f32 and the CsRankWorkspace /
// RollingIcWorkspace handles, with the same defaults, dtype gates (strict f32
// for rank ops, f32/f64 for IC and stock correlation, bool/uint8 masks) and
// error mapping (negative status -> ValueError, positive -> RuntimeError).
// All compute goes through libfcb200.so (include/fcb200.h); the GIL is
// released around every call.  f32 inputs of rolling_ic / stock_corr are
// passed at their own width (the kernels widen them exactly), which gives the
// same results as the reference's host-side f32->f64 upcast.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fcb200.h"

namespace py = pybind11;

using ArrF32 = py::array_t<float, py::array::c_style>;
using ArrF64 = py::array_t<double, py::array::c_style>;
using ArrU8 = py::array_t<uint8_t, py::array::c_style | py::array::forcecast>;

namespace {

struct Workspace {
  fcb_workspace* ws;
  Workspace() : ws(fcb_workspace_create()) {
    if (ws == nullptr) throw std::bad_alloc();
  }
  ~Workspace() { fcb_workspace_destroy(ws); }
  Workspace(const Workspace&) = delete;
  Workspace& operator=(const Workspace&) = delete;
  void clear() { fcb_workspace_clear(ws); }
};
struct CsRankWorkspace : Workspace {};
struct RollingIcWorkspace : Workspace {};

void require_ndarray(py::handle obj, const char* name) {
  if (!py::isinstance<py::array>(obj)) throw py::type_error(std::string(name) + " must be a numpy array");
}

py::dtype dtype_of(py::handle obj) { return py::reinterpret_borrow<py::array>(obj).dtype(); }

ArrF32 require_f32(py::handle obj, const char* name) {
  require_ndarray(obj, name);
  if (!(dtype_of(obj) == py::dtype::of<float>()))
    throw py::type_error(std::string(name) + " must be float32 (float64 downcast is adapter responsibility)");
  return py::cast<ArrF32>(obj);
}

// f32 or f64 panel, kept at its own width; returns the dtype code.
py::array float_panel(py::handle obj, const char* name, int& dtype) {
  require_ndarray(obj, name);
  py::dtype dt = dtype_of(obj);
  if (dt == py::dtype::of<float>()) {
    dtype = FCB_DTYPE_F32;
    return py::cast<ArrF32>(obj);
  }
  if (dt == py::dtype::of<double>()) {
    dtype = FCB_DTYPE_F64;
    return py::cast<ArrF64>(obj);
  }
  throw py::type_error(std::string(name) + " must be float32 or float64");
}

const uint8_t* mask_or_null(py::object obj, const char* name, py::ssize_t T, py::ssize_t N, ArrU8& holder) {
  if (obj.is_none()) return nullptr;
  require_ndarray(obj, name);
  py::dtype dt = dtype_of(obj);
  if (!(dt == py::dtype::of<bool>() || dt == py::dtype::of<uint8_t>()))
    throw py::value_error(std::string(name) + " must be bool or uint8");
  holder = py::cast<ArrU8>(obj);
  if (holder.ndim() != 2 || holder.shape(0) != T || holder.shape(1) != N)
    throw std::invalid_argument(std::string(name) + " shape must be (T,N) matching input");
  return holder.data();
}

int require_int(py::handle obj, const char* name) {
  if (!py::isinstance<py::int_>(obj)) throw std::invalid_argument(std::string(name) + " must be an integer");
  return py::cast<int>(obj);
}

void check_rc(int rc, const char* fn) {
  if (rc == 0) return;
  if (rc < 0) throw std::invalid_argument(std::string(fn) + " contract error code " + std::to_string(rc));
  throw std::runtime_error(std::string(fn) + " failed with error code " + std::to_string(rc) + " (" +
                           fcb_status_string(rc) + ")");
}

// The workspace argument must be the handle class the function is bound to
// (CsRankWorkspace for cs_rank / parameter_scan, RollingIcWorkspace for
// rolling_ic); any other object raises TypeError, as a typed pybind11
// parameter would.
template <typename W>
fcb_workspace* ws_ptr(py::object w, const char* expected) {
  if (w.is_none()) return nullptr;
  if (!py::isinstance<W>(w))
    throw py::type_error(std::string("workspace must be a ") + expected + " or None");
  return py::cast<W&>(w).ws;
}

void check_2d(const py::array& a, const char* name, py::ssize_t& T, py::ssize_t& N) {
  if (a.ndim() != 2) throw std::invalid_argument(std::string(name) + " must be 2-D (T,N)");
  T = a.shape(0);
  N = a.shape(1);
  if (T < 1 || N < 1) throw std::invalid_argument(std::string(name) + " must be (T,N) with T,N >= 1");
}

// ---------------------------------------------------------------- cs_rank
py::array_t<float> cs_rank_f32(py::object X, py::object mask, bool descending, py::object workspace) {
  ArrF32 xa = require_f32(X, "X");
  py::ssize_t T, N;
  check_2d(xa, "X", T, N);
  if (N > (1 << 24)) throw std::invalid_argument("N > 2^24 (rank precision cap)");
  if (static_cast<int64_t>(T) * N > INT32_MAX) throw std::invalid_argument("T*N exceeds INT32_MAX (implementation cap)");
  ArrU8 mh;
  const uint8_t* mp = mask_or_null(mask, "mask", T, N, mh);
  fcb_workspace* ws = ws_ptr<CsRankWorkspace>(workspace, "CsRankWorkspace");
  py::array_t<float> out({T, N});
  float* op = out.mutable_data();
  const float* xp = xa.data();
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = fcb_cs_rank_f32(xp, mp, static_cast<int>(T), static_cast<int>(N), descending ? 1 : 0, op, ws);
  }
  check_rc(rc, "cs_rank_gpu");
  return out;
}

// ----------------------------------------------------------- rolling_ic
py::object rolling_ic_f64(py::object F, py::object R, py::object fmask, py::object rmask, py::object min_valid_obj,
                          bool return_ranks, py::object workspace) {
  int fdt = 0, rdt = 0;
  py::array fa = float_panel(F, "F", fdt);
  py::array ra = float_panel(R, "R", rdt);
  py::ssize_t T, N;
  check_2d(fa, "F", T, N);
  if (ra.ndim() != 2 || ra.shape(0) != T || ra.shape(1) != N) throw std::invalid_argument("R shape must match F (T,N)");
  if (static_cast<int64_t>(T) * N > INT32_MAX) throw std::invalid_argument("T*N exceeds INT32_MAX (implementation cap)");
  const int min_valid = require_int(min_valid_obj, "min_valid");
  if (min_valid < 2) throw std::invalid_argument("min_valid must be >= 2");
  ArrU8 fh, rh;
  const uint8_t* fmp = mask_or_null(fmask, "fmask", T, N, fh);
  const uint8_t* rmp = mask_or_null(rmask, "rmask", T, N, rh);
  fcb_workspace* ws = ws_ptr<RollingIcWorkspace>(workspace, "RollingIcWorkspace");
  py::array_t<double> ic({T});
  py::array_t<double> rf, rr;
  double *rfp = nullptr, *rrp = nullptr;
  if (return_ranks) {
    rf = py::array_t<double>({T, N});
    rr = py::array_t<double>({T, N});
    rfp = rf.mutable_data();
    rrp = rr.mutable_data();
  }
  double* icp = ic.mutable_data();
  const void* fp = fa.data();
  const void* rp = ra.data();
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = fcb_rolling_ic(fp, fdt, rp, rdt, fmp, rmp, static_cast<int>(T), static_cast<int>(N), min_valid, icp, rfp,
                        rrp, ws);
  }
  check_rc(rc, "rolling_ic_gpu");
  if (!return_ranks) return ic;
  return py::make_tuple(ic, rf, rr);
}

// ----------------------------------------------------------- stock_corr
py::object stock_corr_f64(py::object X, py::object mask, bool return_stats) {
  int dt = 0;
  py::array xa = float_panel(X, "X", dt);
  py::ssize_t T, N;
  check_2d(xa, "X", T, N);
  if (static_cast<int64_t>(T) * N > INT32_MAX) throw std::invalid_argument("T*N exceeds INT32_MAX (implementation cap)");
  if (static_cast<int64_t>(N) * N > INT32_MAX)
    throw std::invalid_argument("N*N exceeds INT32_MAX (output grid cap, N <= 46340)");
  ArrU8 mh;
  const uint8_t* mp = mask_or_null(mask, "mask", T, N, mh);
  py::array_t<double> out({N, N});
  double* op = out.mutable_data();
  const void* xp = xa.data();
  int path = -1, fb = 0;
  int rc;
  {
    py::gil_scoped_release nogil;
    rc = fcb_stock_corr(xp, dt, mp, static_cast<int>(T), static_cast<int>(N), op, &path, &fb);
  }
  if (rc == FCB_ERR_CAP4)
    throw std::invalid_argument(
        "correlation domain violation: max|x| > 1e150 or a nonzero |x| < 1e-150 on a valid cell");
  check_rc(rc, "stock_corr_gpu");
  if (!return_stats) return out;
  py::dict sd;
  sd["selected_path"] = path;
  sd["fallback_count"] = fb;
  return py::make_tuple(out, sd);
}

// -------------------------------------------------------- parameter_scan
py::dict parameter_scan_f32(py::object X, py::object mask, bool return_timing, py::object active_groups,
                            py::object workspace) {
  ArrF32 xa = require_f32(X, "X");
  py::ssize_t T, N;
  check_2d(xa, "X", T, N);
  if (N > (1 << 24)) throw std::invalid_argument("N > 2^24 (rank precision cap)");
  const int64_t total = static_cast<int64_t>(T) * N;
  if (total > INT32_MAX) throw std::invalid_argument("T*N exceeds INT32_MAX (implementation cap)");
  int act[4] = {1, 1, 1, 1};
  int nact = 4;
  if (!active_groups.is_none()) {
    py::sequence seq = py::cast<py::sequence>(active_groups);
    if (py::len(seq) != 4) throw std::invalid_argument("active_groups must have length 4");
    nact = 0;
    for (int g = 0; g < 4; ++g) {
      const int v = py::cast<int>(seq[g]);
      if (v != 0 && v != 1) throw std::invalid_argument("active_groups values must be 0 or 1");
      act[g] = v;
      nact += v;
    }
  }
  const bool need_mask = act[0] || act[2];
  ArrU8 mh;
  const uint8_t* mp = nullptr;
  if (need_mask) {
    if (mask.is_none()) throw std::invalid_argument("parameter_scan requires a mask when any masked group is active");
    mp = mask_or_null(mask, "mask", T, N, mh);
  }
  if (static_cast<size_t>(nact) * static_cast<size_t>(total) * sizeof(float) > (4ull << 30))
    throw std::invalid_argument("active*T*N*4 bytes exceeds the host output budget");
  fcb_workspace* ws = ws_ptr<CsRankWorkspace>(workspace, "CsRankWorkspace");
  py::array_t<float> outs[4];
  float* op[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int g = 0; g < 4; ++g)
    if (act[g]) {
      outs[g] = py::array_t<float>({T, N});
      op[g] = outs[g].mutable_data();
    }
  int status[4];
  double tms[4];
  float tgms[4];
  const float* xp = xa.data();
  double elapsed = 0.0;
  int rc;
  {
    py::gil_scoped_release nogil;
    const auto t0 = std::chrono::steady_clock::now();
    rc = fcb_parameter_scan_f32(xp, mp, static_cast<int>(T), static_cast<int>(N), op, status,
                                return_timing ? tms : nullptr, return_timing ? tgms : nullptr, act, ws);
    elapsed = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  check_rc(rc, "parameter_scan_gpu");
  py::dict result;
  py::list groups, st;
  for (int g = 0; g < 4; ++g) {
    st.append(status[g]);
    if (status[g] == 0) {
      groups.append(outs[g]);
    } else if (status[g] == 9 || status[g] == 701 || status[g] == FCB_GROUP_NOT_EXECUTED) {
      groups.append(py::none());
    } else {
      throw std::runtime_error("parameter_scan_gpu group-level error code " + std::to_string(status[g]));
    }
  }
  result["groups"] = groups;
  result["group_status"] = st;
  if (return_timing) {
    py::list a, b;
    for (int g = 0; g < 4; ++g) {
      a.append(tms[g]);
      b.append(tgms[g]);
    }
    result["time_ms"] = a;
    result["time_gpu_ms"] = b;
    result["_elapsed_ms_diag"] = elapsed;
  }
  return result;
}

}  // namespace

PYBIND11_MODULE(factor_cuda_pybind, m) {
  m.doc() =
      "B200 (sm_100a) drop-in for factor-cuda's factor_cuda_pybind module.\n"
      "  cs_rank_f32(X, mask=None, descending=False, workspace=None) -> (T,N) f32\n"
      "  rolling_ic_f64(F, R, fmask=None, rmask=None, min_valid=30,\n"
      "                 return_ranks=False, workspace=None) -> (T,) f64 | (ic, rf, rr)\n"
      "  stock_corr_f64(X, mask=None, return_stats=False) -> (N,N) f64\n"
      "  parameter_scan_f32(X, mask, return_timing=False, active_groups=None,\n"
      "                     workspace=None) -> {groups, group_status, ...}\n"
      "  CsRankWorkspace() / RollingIcWorkspace(): cached device buffers, .clear().\n"
      "Compute runs in libfcb200.so (C ABI, include/fcb200.h).";
  py::class_<Workspace>(m, "_Workspace").def("clear", &Workspace::clear);
  py::class_<CsRankWorkspace, Workspace>(m, "CsRankWorkspace")
      .def(py::init<>())
      .def("clear", &CsRankWorkspace::clear, "Release all cached device buffers (idempotent).");
  py::class_<RollingIcWorkspace, Workspace>(m, "RollingIcWorkspace")
      .def(py::init<>())
      .def("clear", &RollingIcWorkspace::clear, "Release all cached device buffers (idempotent).");
  m.def("cs_rank_f32", &cs_rank_f32, py::arg("X"), py::arg("mask") = py::none(), py::arg("descending") = false,
        py::arg("workspace") = py::none(),
        "Stable ordinal cross-sectional rank of a (T,N) float32 panel; invalid -> NaN 0x7fc00000.");
  m.def("rolling_ic_f64", &rolling_ic_f64, py::arg("F"), py::arg("R"), py::arg("fmask") = py::none(),
        py::arg("rmask") = py::none(), py::arg("min_valid") = 30, py::arg("return_ranks") = false,
        py::arg("workspace") = py::none(), "Daily cross-sectional Spearman IC.");
  m.def("stock_corr_f64", &stock_corr_f64, py::arg("X"), py::arg("mask") = py::none(),
        py::arg("return_stats") = false, "(N,N) pairwise-complete stock correlation matrix.");
  m.def("parameter_scan_f32", &parameter_scan_f32, py::arg("X"), py::arg("mask"), py::arg("return_timing") = false,
        py::arg("active_groups") = py::none(), py::arg("workspace") = py::none(),
        "G=4 rank parameter scan (direction x mask_mode), one fused pass.");
}
