// Kokkos-API host shim (oracle test infrastructure): real math wrappers.
// Each forwards to the C library routine of the same name.
#pragma once

#include <cmath>
#include <type_traits>

#include "Kokkos_Complex.hpp"

namespace Kokkos {

using std::acos;
using std::asin;
using std::atan;
using std::atan2;
using std::cbrt;
using std::ceil;
using std::cos;
using std::cosh;
using std::exp;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::hypot;
using std::log;
using std::pow;
using std::round;
using std::sin;
using std::sinh;
using std::sqrt;
using std::tan;
using std::tanh;

template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
constexpr T abs(const T value) noexcept {
  return value < T(0) ? -value : value;
}
template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
bool isfinite(const T value) noexcept {
  return std::isfinite(value);
}
template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
bool isnan(const T value) noexcept {
  return std::isnan(value);
}
template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
bool isinf(const T value) noexcept {
  return std::isinf(value);
}

}  // namespace Kokkos
