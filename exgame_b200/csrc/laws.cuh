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
// 6-axis slice of the 24-axis Jacobian per evaluation).
#pragma once
#include "geom.cuh"

namespace exg {

enum : int { LAW_SIMPLE = 0, LAW_CRITICAL = 1, LAW_PERPENDICULAR = 2, LAW_TORSIONAL = 3 };

template <class S>
EXG_HD void law_axial(int law, const double* prm, const S* ma, const S* mb, const S* ta, const S* tb, double dt, double warp,
                      S* wa) {
  S la[3] = {S(prm[0]), S(prm[1]), S(prm[2])};
  S lb[3] = {S(prm[3]), S(prm[4]), S(prm[5])};
  S pa[4], pb[4], line[6];
  anchor_point(ma, la, pa);
  anchor_point(mb, lb, pb);
  point_join(pa, pb, line);
  S d = soft_weight_norm(line, S(prm[9]));
  S raw[6], unit[6], rel[6];
  wrench_from_line(line, raw);
  S inv_d = S(1.0) / d;
#pragma unroll
  for (int i = 0; i < 6; ++i) { unit[i] = raw[i] * inv_d; rel[i] = ta[i] - tb[i]; }
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

template <class S>
EXG_HD void law_perpendicular(const double* prm, const S* ma, const S* mb, const S* ta, const S* tb, double warp, S* wa) {
  S zero[3] = {S(0.0), S(0.0), S(0.0)};
  S pa[4], pb[4], line[6];
  anchor_point(ma, zero, pa);
  anchor_point(mb, zero, pb);
  point_join(pa, pb, line);
  S d = soft_weight_norm(line, S(prm[1]));
  S b_eff = S(prm[0] / (warp * warp));
  S dir[3], n[3];
  line_direction(line, dir);
  S inv_d = S(1.0) / d;
#pragma unroll
  for (int i = 0; i < 3; ++i) n[i] = dir[i] * inv_d;
  S rel[6], v[3];
#pragma unroll
  for (int i = 0; i < 6; ++i) rel[i] = ta[i] - tb[i];
  velocity_at(rel, pa, v);
  S vn = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
  S ca[3], tip[3];
  point_coords(pa, ca);
#pragma unroll
  for (int i = 0; i < 3; ++i) tip[i] = ca[i] + (v[i] - n[i] * vn) * (-b_eff);
  S pt[4], l2[6];
  point_make(tip, pt);
  point_join(pt, pa, l2);
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

template <class S>
EXG_HD void law_wrench(int law, const double* prm, const S* ma, const S* mb, const S* ta, const S* tb, double dt, double warp,
                       S* wa) {
  if (law <= LAW_CRITICAL) law_axial(law, prm, ma, mb, ta, tb, dt, warp, wa);
  else if (law == LAW_PERPENDICULAR) law_perpendicular(prm, ma, mb, ta, tb, warp, wa);
  else law_torsional(prm, ta, tb, warp, wa);
}

}  // namespace exg
