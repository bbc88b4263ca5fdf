// ORACLE — test infrastructure only (CPU restatement the CUDA path is checked against).
//
// Scalar carriers: f64 / f32, and a first-order forward-AD number Dual<N, R> restating
// `Tangent<N, R>` (crates/clifford/src/tangent.rs:160-305): value + N partials, chain
// rule per transcendental. The Study-form transcendentals and their effective-zero
// seams follow crates/peano/src/scalar.rs:67-131 with the thresholds of
// crates/peano/src/support.rs:39-49 (|x| < 1e-9 for f64, < 1e-5 for f32), chosen by the
// carrier's standard part (support.rs:24-37).
#pragma once
#include <cmath>
#include "pga3.hpp"

namespace oracle {

inline bool eff_zero(double x) { return std::fabs(x) < 1e-9; }
inline bool eff_zero(float x) { return std::fabs(x) < 1e-5f; }

template <int N, class R>
struct Dual {
  R v;
  R g[N];
  Dual() : v(R(0)) { for (int i = 0; i < N; ++i) g[i] = R(0); }
  Dual(double x) : v(R(x)) { for (int i = 0; i < N; ++i) g[i] = R(0); }
  static Dual seed(R value, int axis) { Dual d; d.v = value; d.g[axis] = R(1); return d; }
  Dual operator+(const Dual& o) const { Dual r; r.v = v + o.v; for (int i = 0; i < N; ++i) r.g[i] = g[i] + o.g[i]; return r; }
  Dual operator-(const Dual& o) const { Dual r; r.v = v - o.v; for (int i = 0; i < N; ++i) r.g[i] = g[i] - o.g[i]; return r; }
  Dual operator-() const { Dual r; r.v = -v; for (int i = 0; i < N; ++i) r.g[i] = -g[i]; return r; }
  Dual operator*(const Dual& o) const {
    Dual r; r.v = v * o.v;
    for (int i = 0; i < N; ++i) r.g[i] = g[i] * o.v + v * o.g[i];
    return r;
  }
  // tangent.rs:171-173, 219-225: a / b = a * recip(b), recip' = -v^2
  Dual recip() const { Dual r; R iv = R(1) / v; r.v = iv; for (int i = 0; i < N; ++i) r.g[i] = g[i] * (-(iv * iv)); return r; }
  // The value is a true quotient, so a dual evaluation's value equals the plain evaluation bit
  // for bit (the reference requires that of its Jacobian and plain kernels,
  // crates/newton/src/accelerator/mod.rs:1410-1492); the partials follow (a'b - ab')/b^2.
  Dual operator/(const Dual& o) const {
    Dual r; r.v = v / o.v;
    R inv = R(1) / o.v;
    for (int i = 0; i < N; ++i) r.g[i] = (g[i] - r.v * o.g[i]) * inv;
    return r;
  }
  Dual scale_grad(R s) const { Dual r; r.v = v; for (int i = 0; i < N; ++i) r.g[i] = g[i] * s; return r; }
};
template <int N, class R> inline bool structurally_zero_dual(const Dual<N, R>& x) {
  if (x.v != R(0)) return false;
  for (int i = 0; i < N; ++i) if (x.g[i] != R(0)) return false;
  return true;
}
template <> inline bool structurally_zero<Dual<24, double>>(const Dual<24, double>& x) { return structurally_zero_dual(x); }
template <> inline bool structurally_zero<Dual<6, double>>(const Dual<6, double>& x) { return structurally_zero_dual(x); }
template <> inline bool structurally_zero<Dual<1, double>>(const Dual<1, double>& x) { return structurally_zero_dual(x); }
template <> inline bool structurally_zero<Dual<24, float>>(const Dual<24, float>& x) { return structurally_zero_dual(x); }

// ── scalar primitive dispatch ───────────────────────────────────────────────
inline double std_part(double x) { return x; }
inline float std_part(float x) { return x; }
template <int N, class R> inline R std_part(const Dual<N, R>& x) { return x.v; }

inline double s_sqrt(double x) { return std::sqrt(x); }
inline float s_sqrt(float x) { return std::sqrt(x); }
inline double s_sin(double x) { return std::sin(x); }
inline float s_sin(float x) { return std::sin(x); }
inline double s_cos(double x) { return std::cos(x); }
inline float s_cos(float x) { return std::cos(x); }
inline double s_exp(double x) { return std::exp(x); }
inline float s_exp(float x) { return std::exp(x); }
inline double s_ln(double x) { return std::log(x); }
inline float s_ln(float x) { return std::log(x); }
inline double s_atan2(double y, double x) { return std::atan2(y, x); }
inline float s_atan2(float y, float x) { return std::atan2(y, x); }
inline double s_powf(double x, double n) { return std::pow(x, n); }
inline float s_powf(float x, float n) { return std::pow(x, n); }

// tangent.rs:257-264
template <int N, class R> inline Dual<N, R> s_sqrt(const Dual<N, R>& a) {
  R val = s_sqrt(a.v); R d = R(1) / (val + val);
  Dual<N, R> r = a.scale_grad(d); r.v = val; return r;
}
template <int N, class R> inline Dual<N, R> s_sin(const Dual<N, R>& a) {
  Dual<N, R> r = a.scale_grad(s_cos(a.v)); r.v = s_sin(a.v); return r;
}
template <int N, class R> inline Dual<N, R> s_cos(const Dual<N, R>& a) {
  Dual<N, R> r = a.scale_grad(-s_sin(a.v)); r.v = s_cos(a.v); return r;
}
template <int N, class R> inline Dual<N, R> s_exp(const Dual<N, R>& a) {
  R val = s_exp(a.v); Dual<N, R> r = a.scale_grad(val); r.v = val; return r;
}
template <int N, class R> inline Dual<N, R> s_ln(const Dual<N, R>& a) {
  Dual<N, R> r = a.scale_grad(R(1) / a.v); r.v = s_ln(a.v); return r;
}
// tangent.rs:282-289
template <int N, class R> inline Dual<N, R> s_atan2(const Dual<N, R>& y, const Dual<N, R>& x) {
  R inv = R(1) / (x.v * x.v + y.v * y.v);
  Dual<N, R> r; r.v = s_atan2(y.v, x.v);
  for (int i = 0; i < N; ++i) r.g[i] = y.g[i] * (x.v * inv) - x.g[i] * (y.v * inv);
  return r;
}
// tangent.rs:279-281
template <int N, class R> inline Dual<N, R> s_powf(const Dual<N, R>& a, const Dual<N, R>& n) { return s_exp(n * s_ln(a)); }

// powi by square-and-multiply (tangent.rs:290-305); the same for plain floats.
template <class T> inline T s_powi(T x, int n) {
  if (n < 0) return s_powi(T(1.0) / x, -n);
  T result = T(1.0), base = x;
  unsigned e = unsigned(n);
  while (e > 0) { if (e & 1) result = result * base; base = base * base; e >>= 1; }
  return result;
}
template <class T> inline T s_max(T a, T b) { return std_part(a) >= std_part(b) ? a : b; }

// ── Study-form transcendentals (crates/peano/src/scalar.rs:67-131) ─────────
template <class T> inline bool seam_zero(const T& x) { return eff_zero(std_part(x)); }

template <class T> inline T sinc_sq(const T& u) {
  if (seam_zero(u))
    return T(1.0) - u * (T(1.0 / 6.0) - u * (T(1.0 / 120.0) - u * T(1.0 / 5040.0)));
  T l = s_sqrt(u);
  return s_sin(l) / l;
}
template <class T> inline T cos_sq(const T& u) {
  if (seam_zero(u))
    return T(1.0) - u * (T(1.0 / 2.0) - u * (T(1.0 / 24.0) - u * T(1.0 / 720.0)));
  return s_cos(s_sqrt(u));
}
template <class T> inline T dsinc_sq(const T& u) {
  if (seam_zero(u * T(1.0 / 100000.0)))
    return -T(1.0 / 6.0) + u * (T(1.0 / 60.0) - u * (T(1.0 / 1680.0) - u * T(1.0 / 90720.0)));
  T l = s_sqrt(u);
  return (l * s_cos(l) - s_sin(l)) / (T(2.0) * l * l * l);
}
template <class T> inline T half_angle_sq(const T& a, const T& s2) {
  T delta = T(1.0) - a;
  if (seam_zero(delta))
    return delta * (T(2.0) + delta * (T(1.0 / 3.0) + delta * T(4.0 / 45.0)));
  T l = s_atan2(s_sqrt(s2), a);
  return l * l;
}

}  // namespace oracle
