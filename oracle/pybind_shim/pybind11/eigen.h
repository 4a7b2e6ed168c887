// pybind11 type casters for the oracle's Eigen-API subset: TEST INFRASTRUCTURE ONLY.
//
// The reference's CPU plugin (src/sbh.cpp:2) includes <pybind11/eigen.h>, whose
// casters target real Eigen types.  This header takes its place on the include
// path of the oracle harness only (oracle/Makefile puts this directory before
// pybind11's own include directory), so that src/sbh.cpp compiles unmodified
// against oracle/eigen_shim.  Conversion rules follow pybind11's documented
// behaviour for Eigen arguments: any numeric array is converted (copied) to the
// Eigen scalar type; vectors accept 1-D arrays, matrices 2-D arrays; results
// are returned as new numpy arrays.
#pragma once

#include <Eigen/Core>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

namespace pybind11 {
namespace detail {

template <typename S, int R, int C>
struct type_caster<Eigen::Matrix<S, R, C>> {
  using Type = Eigen::Matrix<S, R, C>;
  PYBIND11_TYPE_CASTER(Type, const_name("numpy.ndarray"));

  bool load(handle src, bool convert) {
    if (!convert && !isinstance<array_t<S>>(src)) return false;
    auto arr = array_t<S, array::forcecast>::ensure(src);
    if (!arr) return false;
    if constexpr (C == 1) {
      ssize_t n;
      if (arr.ndim() == 1) {
        n = arr.shape(0);
      } else if (arr.ndim() == 2 && (arr.shape(0) == 1 || arr.shape(1) == 1)) {
        n = arr.shape(0) * arr.shape(1);
      } else {
        return false;
      }
      if (R != Eigen::Dynamic && n != R) return false;
      auto flat = array_t<S, array::forcecast | array::c_style>::ensure(arr);
      if (!flat) return false;
      assign_vector(value, flat.data(), n);
      return true;
    } else {
    if (arr.ndim() != 2) return false;
    auto c = array_t<S, array::forcecast | array::c_style>::ensure(arr);
    if (!c) return false;
    const ssize_t rows = c.shape(0), cols = c.shape(1);
    value.resize(rows, cols);
    const S* p = c.data();
    for (ssize_t i = 0; i < rows; i++)
      for (ssize_t j = 0; j < cols; j++) value(i, j) = p[i * cols + j];
    return true;
    }
  }

  static handle cast(const Type& m, return_value_policy, handle) {
    if constexpr (C == 1) {
      array_t<S> out(static_cast<ssize_t>(m.size()));
      S* p = out.mutable_data();
      for (ssize_t i = 0; i < static_cast<ssize_t>(m.size()); i++) p[i] = m(i);
      return out.release();
    } else {
    const ssize_t rows = m.rows(), cols = m.cols();
    array_t<S> out({rows, cols});
    S* p = out.mutable_data();
    for (ssize_t i = 0; i < rows; i++)
      for (ssize_t j = 0; j < cols; j++) p[i * cols + j] = m(i, j);
    return out.release();
    }
  }

 private:
  template <int RR = R>
  static void assign_vector(Type& v, const S* p, ssize_t n,
                            typename std::enable_if<RR == Eigen::Dynamic>::type* = nullptr) {
    v.resize(n, 1);
    for (ssize_t i = 0; i < n; i++) v(i) = p[i];
  }
  template <int RR = R>
  static void assign_vector(Type& v, const S* p, ssize_t n,
                            typename std::enable_if<RR != Eigen::Dynamic>::type* = nullptr) {
    for (ssize_t i = 0; i < n; i++) v(i) = p[i];
  }
};

}  // namespace detail
}  // namespace pybind11
