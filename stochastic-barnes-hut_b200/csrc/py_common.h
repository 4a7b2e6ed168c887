// Helpers shared by the pybind11 modules `sbh` and `sbh_gpu`.
#pragma once

#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sbh_b200.h"

namespace sbhpy {

namespace py = pybind11;

// Raises the Python exception that matches an sbh_status.
inline void check(int status) {
  if (status == SBH_OK) return;
  std::string msg = std::string(sbh_status_string(status)) + ": " + sbh_last_error();
  if (status == SBH_ERR_INVALID_ARGUMENT) throw py::value_error(msg);
  if (status == SBH_ERR_OUT_OF_MEMORY) throw std::bad_alloc();
  throw std::runtime_error(msg);
}

using FArrayC = py::array_t<float, py::array::c_style | py::array::forcecast>;
using FArrayF = py::array_t<float, py::array::f_style | py::array::forcecast>;

// Row-major [n][dim] float32 view/copy of an array-like (the pybind11 Eigen
// caster of the reference converts float64 input to float32 the same way).
inline FArrayC as_rows(const py::handle& obj, long long n_expected, int dim, const char* what) {
  FArrayC a = FArrayC::ensure(obj);
  if (!a) throw py::type_error(std::string(what) + " must be a numeric array");
  if (a.ndim() != 2 || a.shape(1) != dim)
    throw py::value_error(std::string(what) + " must have shape (n, " + std::to_string(dim) + ")");
  if (n_expected >= 0 && a.shape(0) != n_expected)
    throw py::value_error(std::string(what) + " has the wrong number of rows");
  return a;
}

inline FArrayC as_vector(const py::handle& obj, long long n, const char* what) {
  FArrayC a = FArrayC::ensure(obj);
  if (!a) throw py::type_error(std::string(what) + " must be a numeric array");
  if (a.size() != n)
    throw py::value_error(std::string(what) + " must have " + std::to_string(n) + " entries");
  return a;
}

// Queries as structure-of-arrays: a Fortran-ordered (n, dim) float32 array is
// x[0..n), y[0..n), z[0..n) in memory, the layout of the C ABI.
inline FArrayF as_queries(const py::handle& obj, int dim) {
  // A C-ordered (n, dim) float64 array -- what the reference's callers pass
  // (python/example.py builds its query grids in NumPy's default float64) --
  // is converted to structure-of-arrays float32 by several threads with the
  // GIL released; anything else goes through NumPy's own conversion.
  if (py::isinstance<py::array_t<double>>(obj)) {
    auto d = py::reinterpret_borrow<py::array>(obj);
    if (d.ndim() == 2 && d.shape(1) == dim && (d.flags() & py::array::c_style)) {
      const long long n = d.shape(0);
      FArrayF a({(py::ssize_t)n, (py::ssize_t)dim});
      const double* src = static_cast<const double*>(d.data());
      float* dst = a.mutable_data();
      {
        py::gil_scoped_release nogil;
        const long long per = 1 << 16;
        const int nt = (int)std::min<long long>(
            std::max(1u, std::thread::hardware_concurrency()), (n + per - 1) / per);
        auto work = [&](int w) {
          const long long b = n * w / nt, e = n * (w + 1) / nt;
          for (int k = 0; k < dim; k++)
            for (long long i = b; i < e; i++) dst[k * n + i] = (float)src[i * dim + k];
        };
        std::vector<std::thread> th;
        for (int w = 1; w < nt; w++) th.emplace_back(work, w);
        if (nt > 0) work(0);
        for (auto& x : th) x.join();
      }
      return a;
    }
  }
  FArrayF a = FArrayF::ensure(obj);
  if (!a) throw py::type_error("queries must be a numeric array");
  if (a.ndim() != 2 || a.shape(1) != dim)
    throw py::value_error("queries must have shape (n, " + std::to_string(dim) + ")");
  return a;
}

}  // namespace sbhpy
