// ORACLE — test infrastructure only (CPU restatement the CUDA path is checked against).
//
// The joint force laws as pure world-frame functions (poses, world twists, epoch) ->
// [wrench on a, wrench on b], scalar-generic so the same source gives the value (S = f64)
// and the 24-axis Jacobian (S = Dual<24, f64>):
//   * axial spring-damper, joints/src/axial_spring_damper/mod.rs:315-385, with the force
//     expressions SimpleSpringDamper (mod.rs:46-58 default) and CriticallyDampedWarped
//     (critically_damped_warped.rs:58-88);
//   * PerpendicularDamperWarped, joints/src/perpendicular_damper_warped.rs:107-162;
//   * TorsionalDamperWarped, joints/src/torsional_damper_warped.rs:93-123.
// Parameter order per law follows each law's `params()` (mod.rs:228-260, etc.).
#pragma once
#include "geom.hpp"

namespace oracle {

enum Law { SIMPLE_SPRING_DAMPER = 0, CRITICALLY_DAMPED_WARPED = 1, PERPENDICULAR_DAMPER_WARPED = 2, TORSIONAL_DAMPER_WARPED = 3 };
inline int law_n_params(int law) { return law <= 1 ? 10 : (law == 2 ? 2 : 1); }

template <class S>
struct WrenchPair { Wrench<S> a, b; };

// critically_damped_warped.rs:58-68 (Padé step)
template <class S> inline S crit_calculate(S c0, S x, S v, S rest, S dt) {
  S omega_0 = s_sqrt(c0);
  S omega_02 = c0;
  return (omega_02 * (x - rest) + (S(1.0) + S(1.0)) * omega_0 * v + omega_02 * dt * v) /
         s_powi(S(1.0) + omega_0 * dt, 2);
}

template <class S>
WrenchPair<S> axial_wrench(int law, const double* p, const Motor<S>& pose_a, const Motor<S>& pose_b,
                           const Twist<S>& vel_a, const Twist<S>& vel_b, double dt, double warp) {
  V3<S> a_local{S(p[0]), S(p[1]), S(p[2])};
  V3<S> b_local{S(p[3]), S(p[4]), S(p[5])};
  S rest{p[6]}, k{p[7]}, c{p[8]}, soft{p[9]};
  Point<S> pa = anchor_point(pose_a, a_local);
  Point<S> pb = anchor_point(pose_b, b_local);
  M<S> line = pa.join(pb);
  S d = soft_weight_norm(line, soft);
  Wrench<S> raw = from_line(line);
  Wrench<S> unit = raw.scale(S(1.0) / d);
  S d_dot = power(unit, vel_a - vel_b);
  S f;
  if (law == SIMPLE_SPRING_DAMPER) {
    f = k * (d - rest) + c * d_dot;
  } else {
    S w(warp);
    S c0 = k / s_powi(w, 2);
    f = crit_calculate(c0, d, d_dot, rest, S(dt));
  }
  Wrench<S> w = unit.scale(-f);
  return {w, -w};
}

template <class S>
WrenchPair<S> perpendicular_wrench(const double* p, const Motor<S>& pose_a, const Motor<S>& pose_b,
                                   const Twist<S>& vel_a, const Twist<S>& vel_b, double warp) {
  Point<S> pa = anchor_point(pose_a, V3<S>());
  Point<S> pb = anchor_point(pose_b, V3<S>());
  M<S> line = pa.join(pb);
  S d = soft_weight_norm(line, S(p[1]));
  S w(warp);
  S b_eff = S(p[0]) / s_powi(w, 2);
  V3<S> dir = line_direction(line);
  S inv_d = S(1.0) / d;
  V3<S> n = dir.scale(inv_d);
  V3<S> v_rel = velocity_at(vel_a - vel_b, pa);
  S v_dot_n = v_rel.dot(n);
  V3<S> v_perp = v_rel - n.scale(v_dot_n);
  V3<S> f = v_perp.scale(-b_eff);
  V3<S> ca = pa.coords();
  Point<S> tip = Point<S>::at(ca + f);
  Wrench<S> wa = from_line(tip.join(pa));
  return {wa, -wa};
}

template <class S>
WrenchPair<S> torsional_wrench(const double* p, const Twist<S>& vel_a, const Twist<S>& vel_b, double warp) {
  V3<S> w_rel = (vel_a - vel_b).ang();
  S w(warp);
  S b_eff = S(p[0]) / s_powi(w, 2);
  Wrench<S> couple = Wrench<S>::make(V3<S>(), w_rel.scale(-b_eff));
  return {couple, -couple};
}

template <class S>
WrenchPair<S> law_wrench(int law, const double* p, const Motor<S>& pose_a, const Motor<S>& pose_b,
                         const Twist<S>& vel_a, const Twist<S>& vel_b, double dt, double warp) {
  switch (law) {
    case SIMPLE_SPRING_DAMPER:
    case CRITICALLY_DAMPED_WARPED: return axial_wrench(law, p, pose_a, pose_b, vel_a, vel_b, dt, warp);
    case PERPENDICULAR_DAMPER_WARPED: return perpendicular_wrench(p, pose_a, pose_b, vel_a, vel_b, warp);
    default: return torsional_wrench(p, vel_a, vel_b, warp);
  }
}

// Potential energy of the axial spring (mod.rs:390-415, default ½k(d-L0)²); the dampers
// have none (lib.rs:236-243).
inline double law_potential(int law, const double* p, const Motor<double>& pose_a, const Motor<double>& pose_b) {
  if (law > 1) return 0.0;
  Point<double> pa = anchor_point(pose_a, V3<double>(p[0], p[1], p[2]));
  Point<double> pb = anchor_point(pose_b, V3<double>(p[3], p[4], p[5]));
  double d = soft_weight_norm(pa.join(pb), p[9]);
  double dl = d - p[6];
  return 0.5 * p[7] * dl * dl;
}

// Plain value kernel (crates/newton/build.rs:938-973): the 12 wrench components
// [fa, ta, fb, tb] at (pose = base, world twists).
inline void plain_eval(int law, const double* p, const double pose_a[8], const double pose_b[8],
                       const double vel_a[6], const double vel_b[6], double dt, double warp, double out[12]) {
  Motor<double> ma = Motor<double>::from_components(pose_a);
  Motor<double> mb = Motor<double>::from_components(pose_b);
  WrenchPair<double> w = law_wrench(law, p, ma, mb, Twist<double>::from6(vel_a), Twist<double>::from6(vel_b), dt, warp);
  w.a.to6(out);
  w.b.to6(out + 6);
}

// Jacobian kernel (crates/newton/build.rs:673-768 = Differential::jacobian,
// crates/clifford/src/pga3/ad.rs:119-150): pose = exp(delta) * base (compose with the
// unit retraction Motor::exp, no half), velocity = value + unit partial. Axis layout:
// pose A 0..6, pose B 6..12, vel A 12..18, vel B 18..24; each block lin xyz then ang xyz.
// Output: 12 components x [value, d/dx0 .. d/dx23] (300 doubles).
inline void jacobian_eval(int law, const double* p, const double pose_a[8], const double pose_b[8],
                          const double vel_a[6], const double vel_b[6], double dt, double warp, double out[300]) {
  using D = Dual<24, double>;
  auto base = [](const double* c) {
    D comps[8];
    for (int i = 0; i < 8; ++i) comps[i] = D(c[i]);
    return Motor<D>::from_components(comps);
  };
  auto dtwist = [](int off) {
    V3<D> l(D::seed(0.0, off), D::seed(0.0, off + 1), D::seed(0.0, off + 2));
    V3<D> a(D::seed(0.0, off + 3), D::seed(0.0, off + 4), D::seed(0.0, off + 5));
    return Twist<D>::make(l, a);
  };
  auto vtwist = [](const double* v, int off) {
    V3<D> l(D::seed(v[0], off), D::seed(v[1], off + 1), D::seed(v[2], off + 2));
    V3<D> a(D::seed(v[3], off + 3), D::seed(v[4], off + 4), D::seed(v[5], off + 5));
    return Twist<D>::make(l, a);
  };
  Motor<D> ma = base(pose_a).compose(motor_exp(dtwist(0)));
  Motor<D> mb = base(pose_b).compose(motor_exp(dtwist(6)));
  Twist<D> va = vtwist(vel_a, 12), vb = vtwist(vel_b, 18);
  WrenchPair<D> w = law_wrench(law, p, ma, mb, va, vb, dt, warp);
  D comps[12];
  w.a.to6(comps);
  w.b.to6(comps + 6);
  for (int c = 0; c < 12; ++c) {
    out[c * 25] = comps[c].v;
    for (int k = 0; k < 24; ++k) out[c * 25 + 1 + k] = comps[c].g[k];
  }
}

}  // namespace oracle
