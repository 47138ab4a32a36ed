// getm_tangent.hpp -- TEST INFRASTRUCTURE ONLY.
//
// Forward-mode (tangent-linear) derivative of the oracle's tracer step: a dual number carries a
// value and one directional derivative through the unchanged templates of getm_oracle.hpp.
// Comparisons and branches act on the value, so every limiter branch is the one the plain FP64
// step takes, and the derivative is that of the discrete step with those branches -- the
// quantity the GPU adjoint's gradient must reproduce (<grad, dx> = tangent(dx)).
#pragma once
#include <cmath>

namespace gor {

struct Dual {
  double v = 0.0, d = 0.0;
  Dual() = default;
  Dual(double x) : v(x), d(0.0) {}  // NOLINT: literals and constants enter as constants
  Dual(double x, double dx) : v(x), d(dx) {}
  Dual& operator+=(const Dual& b) { d += b.d; v += b.v; return *this; }
  Dual& operator-=(const Dual& b) { d -= b.d; v -= b.v; return *this; }
  Dual& operator*=(const Dual& b) { d = d * b.v + v * b.d; v *= b.v; return *this; }
  Dual& operator/=(const Dual& b) {
    const double q = v / b.v;
    d = (d - q * b.d) / b.v;
    v = q;
    return *this;
  }
};

inline Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(const Dual& a, const Dual& b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
inline Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
inline double ceil(const Dual& a) { return std::ceil(a.v); }

}  // namespace gor
