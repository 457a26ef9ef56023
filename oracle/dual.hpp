// ORACLE - test infrastructure only.  Forward-mode dual numbers for the derivative checker: a value
// and its derivatives along K directions, carried through every + - * / sqrt of the restated step
// (solve_stage.cpp's StageT, the narrowphase's collideT).  Nothing in the product uses this.
//
// The derivative of each operation is the exact one of its rounded result's formula; at the
// points where a function has none it takes the same side as the product's reverse-mode replay
// (bearing_b200/csrc/tape.hpp): sqrt at 0 gives 0, |x| at 0 gives 0, atan2 at (0, 0) gives 0, and
// comparisons, min and max follow the values.
#pragma once

#include <cmath>

namespace dual {

constexpr int K = 5;   // friction, restitution, and the three components of a launch velocity

struct D {
  double v = 0;
  double d[K] = {0, 0, 0, 0, 0};
  D() = default;
  D(double x) : v(x) {}   // NOLINT: constants mix freely with dual numbers
};

inline D operator+(const D& a, const D& b) {
  D r(a.v + b.v);
  for (int k = 0; k < K; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
inline D operator-(const D& a, const D& b) {
  D r(a.v - b.v);
  for (int k = 0; k < K; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
inline D operator*(const D& a, const D& b) {
  D r(a.v * b.v);
  for (int k = 0; k < K; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
inline D operator/(const D& a, const D& b) {
  D r(a.v / b.v);
  for (int k = 0; k < K; k++) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
inline D operator-(const D& a) {
  D r(-a.v);
  for (int k = 0; k < K; k++) r.d[k] = -a.d[k];
  return r;
}
inline D& operator+=(D& a, const D& b) { return a = a + b; }
inline D& operator-=(D& a, const D& b) { return a = a - b; }
inline D& operator*=(D& a, const D& b) { return a = a * b; }
inline D& operator/=(D& a, const D& b) { return a = a / b; }

inline bool operator<(const D& a, const D& b) { return a.v < b.v; }
inline bool operator>(const D& a, const D& b) { return a.v > b.v; }
inline bool operator<=(const D& a, const D& b) { return a.v <= b.v; }
inline bool operator>=(const D& a, const D& b) { return a.v >= b.v; }
inline bool operator==(const D& a, const D& b) { return a.v == b.v; }
inline bool operator!=(const D& a, const D& b) { return a.v != b.v; }

inline D sqrt(const D& a) {
  D r(std::sqrt(a.v));
  const double g = r.v > 0 ? 0.5 / r.v : 0.0;
  for (int k = 0; k < K; k++) r.d[k] = a.d[k] * g;
  return r;
}
inline D fabs(const D& a) {
  const double s = a.v < 0 ? -1.0 : a.v > 0 ? 1.0 : 0.0;
  D r(a.v < 0 ? -a.v : a.v);
  for (int k = 0; k < K; k++) r.d[k] = a.d[k] * s;
  return r;
}
inline double val(const D& a) { return a.v; }

// A value computed elsewhere (value r of atan2(y, x)) with its derivatives.
inline D atan2_lift(double r, const D& y, const D& x) {
  D out(r);
  const double den = x.v * x.v + y.v * y.v;
  if (den > 0)
    for (int k = 0; k < K; k++) out.d[k] = (x.v * y.d[k] - y.v * x.d[k]) / den;
  return out;
}

}  // namespace dual
