// The joint force laws as scalar-generic device functions:
//   (pose A, pose B, world twist A, world twist B, dt, warp, params) -> wrench on A (BIV),
// the wrench on B being its negation for every law (third law by construction).
// Restated from the reference's `JointImpl::wrench` implementations:
//   axial spring-damper        crates/joints/src/axial_spring_damper/mod.rs:315-385
//     SimpleSpringDamper       force k(d-L0) + c d'  (mod.rs:46-58)
//     CriticallyDampedWarped   Padé step (critically_damped_warped.rs:58-88)
//   PerpendicularDamperWarped  crates/joints/src/perpendicular_damper_warped.rs:107-162
//   TorsionalDamperWarped      crates/joints/src/torsional_damper_warped.rs:93-123
// Instantiated with S = double (plain f64 path), float (mixed path) and Dual<6, R> (one
// 6-axis slice of the 24-axis Jacobian per evaluation). Law ids from kUserLawFirst on are the
// traced laws of user_laws.cuh, with the same signature.
#pragma once
#include "geom.cuh"

namespace exg {

enum : int { LAW_SIMPLE = 0, LAW_CRITICAL = 1, LAW_PERPENDICULAR = 2, LAW_TORSIONAL = 3 };

// Pose-only intermediates are computed in P and lifted to S where they meet the twists. P = S
// is the plain evaluation and the pose slices of the Jacobian; P = R with S = Dual<N, R> gives the
// twist slices, whose pose chain has no partials, at plain cost (same values: a dual's value part
// is the plain evaluation).
template <class S> struct Lift {
  static EXG_HD S from(const S& x) { return x; }
};
template <int N, class R> struct Lift<Dual<N, R>> {
  static EXG_HD Dual<N, R> from(const Dual<N, R>& x) { return x; }
  static EXG_HD Dual<N, R> from(const R& x) { Dual<N, R> r; r.v = x; return r; }
};

}  // namespace exg
// Laws traced from their scalar-generic form at build time (exgame_b200/viete.py): law ids from
// kUserLawFirst on.
#include "user_laws.cuh"
namespace exg {

template <class S, class P = S>
EXG_HD void law_axial(int law, const double* prm, const P* ma, const P* mb, const S* ta, const S* tb, double dt,
                      double warp, S* wa) {
  P la[3] = {P(prm[0]), P(prm[1]), P(prm[2])};
  P lb[3] = {P(prm[3]), P(prm[4]), P(prm[5])};
  P pa[4], pb[4], line[6];
  anchor_point(ma, la, pa);
  anchor_point(mb, lb, pb);
  point_join(pa, pb, line);
  P dp = soft_weight_norm(line, P(prm[9]));
  P raw[6];
  wrench_from_line(line, raw);
  P inv_d = P(1.0) / dp;
  S unit[6], rel[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) { unit[i] = Lift<S>::from(raw[i] * inv_d); rel[i] = ta[i] - tb[i]; }
  const S d = Lift<S>::from(dp);
  S d_dot = screw_power(unit, rel);
  S f;
  if (law == LAW_SIMPLE) {
    f = S(prm[7]) * (d - S(prm[6])) + S(prm[8]) * d_dot;
  } else {
    S c0 = S(prm[7]) / S(warp * warp);
    S w0 = s_sqrt(c0);
    S h = S(dt);
    S den = S(1.0) + w0 * h;
    f = (c0 * (d - S(prm[6])) + S(2.0) * w0 * d_dot + c0 * h * d_dot) / (den * den);
  }
  S nf = -f;
#pragma unroll
  for (int i = 0; i < 6; ++i) wa[i] = unit[i] * nf;
}

template <class S, class P = S>
EXG_HD void law_perpendicular(const double* prm, const P* ma, const P* mb, const S* ta, const S* tb, double warp,
                              S* wa) {
  P zero[3] = {P(0.0), P(0.0), P(0.0)};
  P pa[4], pb[4], line[6];
  anchor_point(ma, zero, pa);
  anchor_point(mb, zero, pb);
  point_join(pa, pb, line);
  P d = soft_weight_norm(line, P(prm[1]));
  S b_eff = S(prm[0] / (warp * warp));
  P dir[3], cp[3];
  line_direction(line, dir);
  P inv_d = P(1.0) / d;
  point_coords(pa, cp);
  S n[3], ca[3], pas[4];
#pragma unroll
  for (int i = 0; i < 3; ++i) { n[i] = Lift<S>::from(dir[i] * inv_d); ca[i] = Lift<S>::from(cp[i]); }
#pragma unroll
  for (int i = 0; i < 4; ++i) pas[i] = Lift<S>::from(pa[i]);
  S rel[6], v[3];
#pragma unroll
  for (int i = 0; i < 6; ++i) rel[i] = ta[i] - tb[i];
  velocity_at(rel, pas, v);
  S vn = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
  S tip[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) tip[i] = ca[i] + (v[i] - n[i] * vn) * (-b_eff);
  S pt[4], l2[6];
  point_make(tip, pt);
  point_join(pt, pas, l2);
  wrench_from_line(l2, wa);
}

template <class S>
EXG_HD void law_torsional(const double* prm, const S* ta, const S* tb, double warp, S* wa) {
  S rel[6], lin[3], ang[3];
#pragma unroll
  for (int i = 0; i < 6; ++i) rel[i] = ta[i] - tb[i];
  screw_to_phys(rel, lin, ang);
  S k = -S(prm[0] / (warp * warp));
  S zero[3] = {S(0.0), S(0.0), S(0.0)};
  S tq[3] = {ang[0] * k, ang[1] * k, ang[2] * k};
  screw_from_phys(zero, tq, wa);
}

template <class S, class P = S>
EXG_HD void law_wrench(int law, const double* prm, const P* ma, const P* mb, const S* ta, const S* tb, double dt,
                       double warp, S* wa) {
  if (law <= LAW_CRITICAL) law_axial<S, P>(law, prm, ma, mb, ta, tb, dt, warp, wa);
  else if (law == LAW_PERPENDICULAR) law_perpendicular<S, P>(prm, ma, mb, ta, tb, warp, wa);
  else if (law == LAW_TORSIONAL) law_torsional(prm, ta, tb, warp, wa);
  else user_law_wrench<S, P>(law - kUserLawFirst, prm, ma, mb, ta, tb, dt, warp, wa);
}

}  // namespace exg
