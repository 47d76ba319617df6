// Kokkos-API host shim (oracle test infrastructure): complex<T>.
// Written from the public Kokkos::complex interface. Arithmetic is the
// textbook formula for + - *; complex/complex division scales by |c|+|d|
// (declared shim semantics); complex/real divides each part.
#pragma once

#include <cmath>
#include <complex>
#include <ostream>
#include <type_traits>

namespace Kokkos {

template <class RealType>
class complex {
 public:
  using value_type = RealType;

  constexpr complex() noexcept : re_(0), im_(0) {}
  constexpr complex(const RealType re) noexcept : re_(re), im_(0) {}
  constexpr complex(const RealType re, const RealType im) noexcept
      : re_(re), im_(im) {}
  template <class Other,
            class = std::enable_if_t<std::is_convertible_v<Other, RealType>>>
  constexpr complex(const complex<Other>& other) noexcept
      : re_(static_cast<RealType>(other.real())),
        im_(static_cast<RealType>(other.imag())) {}
  complex(const std::complex<RealType>& other) noexcept
      : re_(other.real()), im_(other.imag()) {}

  constexpr RealType& real() noexcept { return re_; }
  constexpr RealType real() const noexcept { return re_; }
  constexpr void real(const RealType value) noexcept { re_ = value; }
  constexpr RealType& imag() noexcept { return im_; }
  constexpr RealType imag() const noexcept { return im_; }
  constexpr void imag(const RealType value) noexcept { im_ = value; }

  constexpr complex& operator=(const RealType value) noexcept {
    re_ = value;
    im_ = 0;
    return *this;
  }
  constexpr complex& operator+=(const complex& o) noexcept {
    re_ += o.re_;
    im_ += o.im_;
    return *this;
  }
  constexpr complex& operator+=(const RealType o) noexcept {
    re_ += o;
    return *this;
  }
  constexpr complex& operator-=(const complex& o) noexcept {
    re_ -= o.re_;
    im_ -= o.im_;
    return *this;
  }
  constexpr complex& operator-=(const RealType o) noexcept {
    re_ -= o;
    return *this;
  }
  constexpr complex& operator*=(const complex& o) noexcept {
    const RealType re = re_ * o.re_ - im_ * o.im_;
    const RealType im = re_ * o.im_ + im_ * o.re_;
    re_ = re;
    im_ = im;
    return *this;
  }
  constexpr complex& operator*=(const RealType o) noexcept {
    re_ *= o;
    im_ *= o;
    return *this;
  }
  complex& operator/=(const complex& y) noexcept {
    const RealType s = std::fabs(y.re_) + std::fabs(y.im_);
    if (s == RealType(0)) {
      re_ /= s;
      im_ /= s;
      return *this;
    }
    const RealType xr = re_ / s;
    const RealType xi = im_ / s;
    const RealType yr = y.re_ / s;
    const RealType yi = -y.im_ / s;
    const RealType denominator = yr * yr + yi * yi;
    re_ = (xr * yr - xi * yi) / denominator;
    im_ = (xr * yi + xi * yr) / denominator;
    return *this;
  }
  constexpr complex& operator/=(const RealType o) noexcept {
    re_ /= o;
    im_ /= o;
    return *this;
  }

 private:
  RealType re_;
  RealType im_;
};

template <class T>
constexpr complex<T> operator+(const complex<T>& x) noexcept {
  return x;
}
template <class T>
constexpr complex<T> operator-(const complex<T>& x) noexcept {
  return complex<T>(-x.real(), -x.imag());
}
template <class T>
constexpr complex<T> operator+(complex<T> x, const complex<T>& y) noexcept {
  return x += y;
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr complex<T> operator+(complex<T> x, const S y) noexcept {
  return x += static_cast<T>(y);
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr complex<T> operator+(const S x, const complex<T>& y) noexcept {
  return complex<T>(static_cast<T>(x) + y.real(), y.imag());
}
template <class T>
constexpr complex<T> operator-(complex<T> x, const complex<T>& y) noexcept {
  return x -= y;
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr complex<T> operator-(complex<T> x, const S y) noexcept {
  return x -= static_cast<T>(y);
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr complex<T> operator-(const S x, const complex<T>& y) noexcept {
  return complex<T>(static_cast<T>(x) - y.real(), -y.imag());
}
template <class T>
constexpr complex<T> operator*(complex<T> x, const complex<T>& y) noexcept {
  return x *= y;
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr complex<T> operator*(complex<T> x, const S y) noexcept {
  return x *= static_cast<T>(y);
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr complex<T> operator*(const S x, const complex<T>& y) noexcept {
  return complex<T>(static_cast<T>(x) * y.real(),
                    static_cast<T>(x) * y.imag());
}
template <class T>
complex<T> operator/(complex<T> x, const complex<T>& y) noexcept {
  return x /= y;
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr complex<T> operator/(complex<T> x, const S y) noexcept {
  return x /= static_cast<T>(y);
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
complex<T> operator/(const S x, const complex<T>& y) noexcept {
  return complex<T>(static_cast<T>(x)) /= y;
}
template <class T>
constexpr bool operator==(const complex<T>& x, const complex<T>& y) noexcept {
  return x.real() == y.real() && x.imag() == y.imag();
}
template <class T>
constexpr bool operator!=(const complex<T>& x, const complex<T>& y) noexcept {
  return !(x == y);
}
template <class T, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
constexpr bool operator==(const complex<T>& x, const S y) noexcept {
  return x.real() == static_cast<T>(y) && x.imag() == T(0);
}

template <class T>
constexpr T real(const complex<T>& x) noexcept {
  return x.real();
}
template <class T>
constexpr T imag(const complex<T>& x) noexcept {
  return x.imag();
}
template <class T>
constexpr complex<T> conj(const complex<T>& x) noexcept {
  return complex<T>(x.real(), -x.imag());
}
template <class T>
T abs(const complex<T>& x) noexcept {
  return std::hypot(x.real(), x.imag());
}
template <class T>
constexpr T norm(const complex<T>& x) noexcept {
  return x.real() * x.real() + x.imag() * x.imag();
}
template <class T>
complex<T> exp(const complex<T>& x) noexcept {
  const T scale = std::exp(x.real());
  return complex<T>(scale * std::cos(x.imag()), scale * std::sin(x.imag()));
}
template <class T>
complex<T> sqrt(const complex<T>& x) noexcept {
  return complex<T>(std::sqrt(std::complex<T>(x.real(), x.imag())));
}
template <class T>
bool isfinite(const complex<T>& x) noexcept {
  return std::isfinite(x.real()) && std::isfinite(x.imag());
}

template <class T>
std::ostream& operator<<(std::ostream& os, const complex<T>& x) {
  return os << '(' << x.real() << ',' << x.imag() << ')';
}

}  // namespace Kokkos
