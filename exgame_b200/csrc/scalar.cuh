// Scalar carriers for the device laws: double, float and the forward-mode dual number
// Dual<N, R> (value + N partials) that gives the force laws' Jacobian blocks. The derivative
// rules are the chain rule per primitive, as the reference's Tangent carrier applies them
// (crates/clifford/src/tangent.rs:160-305). Transcendentals call the CUDA math library on the
// device and libm on the host.
#pragma once
#include <cmath>
#include "pga3.cuh"

namespace exg {

EXG_HD double s_sqrt(double x) { return sqrt(x); }
EXG_HD float s_sqrt(float x) { return sqrtf(x); }
EXG_HD double s_sin(double x) { return sin(x); }
EXG_HD float s_sin(float x) { return sinf(x); }
EXG_HD double s_cos(double x) { return cos(x); }
EXG_HD float s_cos(float x) { return cosf(x); }
EXG_HD double s_atan2(double y, double x) { return atan2(y, x); }
EXG_HD float s_atan2(float y, float x) { return atan2f(y, x); }
EXG_HD double s_exp(double x) { return exp(x); }
EXG_HD float s_exp(float x) { return expf(x); }
EXG_HD double s_log(double x) { return log(x); }
EXG_HD float s_log(float x) { return logf(x); }
EXG_HD double s_abs(double x) { return fabs(x); }
EXG_HD float s_abs(float x) { return fabsf(x); }

template <int N, class R>
struct Dual {
  R v;
  R g[N];
  EXG_HD Dual() : v(R(0)) {
#pragma unroll
    for (int i = 0; i < N; ++i) g[i] = R(0);
  }
  EXG_HD Dual(double x) : v(R(x)) {
#pragma unroll
    for (int i = 0; i < N; ++i) g[i] = R(0);
  }
  EXG_HD Dual operator+(const Dual& o) const {
    Dual r; r.v = v + o.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.g[i] = g[i] + o.g[i];
    return r;
  }
  EXG_HD Dual operator-(const Dual& o) const {
    Dual r; r.v = v - o.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.g[i] = g[i] - o.g[i];
    return r;
  }
  EXG_HD Dual operator-() const {
    Dual r; r.v = -v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.g[i] = -g[i];
    return r;
  }
  EXG_HD Dual operator*(const Dual& o) const {
    Dual r; r.v = v * o.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.g[i] = g[i] * o.v + v * o.g[i];
    return r;
  }
  EXG_HD Dual scaled(R value, R d) const {  // f(x) with f(v) = value, f'(v) = d
    Dual r; r.v = value;
#pragma unroll
    for (int i = 0; i < N; ++i) r.g[i] = g[i] * d;
    return r;
  }
  EXG_HD Dual recip() const { R iv = R(1) / v; return scaled(iv, -(iv * iv)); }
  // true quotient for the value (equals the plain evaluation bit for bit), (a'b - ab')/b^2 for
  // the partials
  EXG_HD Dual operator/(const Dual& o) const {
    Dual r; r.v = v / o.v;
    R inv = R(1) / o.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.g[i] = (g[i] - r.v * o.g[i]) * inv;
    return r;
  }
};

template <int N, class R> struct ScalarTraits<Dual<N, R>> {
  using Real = R;
  static EXG_HD R std_part(const Dual<N, R>& x) { return x.v; }
  static EXG_HD bool eff_zero(const Dual<N, R>& x) { return ScalarTraits<R>::eff_zero(x.v); }
};

template <int N, class R> EXG_HD Dual<N, R> s_sqrt(const Dual<N, R>& a) { R r = s_sqrt(a.v); return a.scaled(r, R(1) / (r + r)); }
template <int N, class R> EXG_HD Dual<N, R> s_sin(const Dual<N, R>& a) { return a.scaled(s_sin(a.v), s_cos(a.v)); }
template <int N, class R> EXG_HD Dual<N, R> s_cos(const Dual<N, R>& a) { return a.scaled(s_cos(a.v), -s_sin(a.v)); }
template <int N, class R> EXG_HD Dual<N, R> s_atan2(const Dual<N, R>& y, const Dual<N, R>& x) {
  R inv = R(1) / (x.v * x.v + y.v * y.v);
  Dual<N, R> r; r.v = s_atan2(y.v, x.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = y.g[i] * (x.v * inv) - x.g[i] * (y.v * inv);
  return r;
}

template <int N, class R> EXG_HD Dual<N, R> s_exp(const Dual<N, R>& a) { R e = s_exp(a.v); return a.scaled(e, e); }
template <int N, class R> EXG_HD Dual<N, R> s_log(const Dual<N, R>& a) { return a.scaled(s_log(a.v), R(1) / a.v); }
// |x| with the derivative sign(x) (0 at x = 0, as the reference's Tangent takes it)
template <int N, class R> EXG_HD Dual<N, R> s_abs(const Dual<N, R>& a) {
  return a.scaled(s_abs(a.v), a.v > R(0) ? R(1) : (a.v < R(0) ? R(-1) : R(0)));
}

template <class S> EXG_HD S sq(const S& x) { return x * x; }
template <class S> EXG_HD bool eff_zero(const S& x) { return ScalarTraits<S>::eff_zero(x); }
template <class S> EXG_HD auto std_part(const S& x) { return ScalarTraits<S>::std_part(x); }

// Study forms: sin(sqrt u)/sqrt u, cos(sqrt u) and d/du of the first, each with its Taylor arm
// near u = 0 (crates/peano/src/scalar.rs:67-131).
template <class S> EXG_HD S sinc_sq(const S& u) {
  if (eff_zero(u)) return S(1.0) - u * (S(1.0 / 6.0) - u * (S(1.0 / 120.0) - u * S(1.0 / 5040.0)));
  S l = s_sqrt(u);
  return s_sin(l) / l;
}
template <class S> EXG_HD S cos_sq(const S& u) {
  if (eff_zero(u)) return S(1.0) - u * (S(0.5) - u * (S(1.0 / 24.0) - u * S(1.0 / 720.0)));
  return s_cos(s_sqrt(u));
}
template <class S> EXG_HD S dsinc_sq(const S& u) {
  if (eff_zero(u * S(1e-5))) return -S(1.0 / 6.0) + u * (S(1.0 / 60.0) - u * (S(1.0 / 1680.0) - u * S(1.0 / 90720.0)));
  S l = s_sqrt(u);
  return (l * s_cos(l) - s_sin(l)) / (S(2.0) * l * l * l);
}

}  // namespace exg
