// Per-body state helpers on the component-major world arrays: pose, body momentum, inertia
// (crates/newton/src/inertia.rs:271-345), body / world velocity and world momentum
// (crates/newton/src/body.rs:141-186), position (body.rs:156-162).
#pragma once
#include "geom.cuh"

namespace exg {

struct BodyView {
  const double* pose;
  const double* mom;
  const double* mass;
  const double* inertia;
  const int* kinematic;
  const int* diagonal;
  int n;
};

template <class S>
EXG_HD void inertia_inverse(const double* I9, bool diag, bool kinematic, double mass, const S* p6, S* v6) {
  if (kinematic) {
#pragma unroll
    for (int c = 0; c < 6; ++c) v6[c] = p6[c];
    return;
  }
  S im = S(1.0 / mass);
  v6[0] = p6[0] * im; v6[1] = p6[1] * im; v6[2] = p6[2] * im;
  if (diag) {
    v6[3] = p6[3] / S(I9[0]); v6[4] = p6[4] / S(I9[4]); v6[5] = p6[5] / S(I9[8]);
  } else {
    const double* a = I9;
    double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    double c10 = a[2] * a[7] - a[1] * a[8], c11 = a[0] * a[8] - a[2] * a[6], c12 = a[1] * a[6] - a[0] * a[7];
    double c20 = a[1] * a[5] - a[2] * a[4], c21 = a[2] * a[3] - a[0] * a[5], c22 = a[0] * a[4] - a[1] * a[3];
    S det = S(a[0] * c00 + a[1] * c01 + a[2] * c02);
    const S* b = p6 + 3;
    v6[3] = (S(c00) * b[0] + S(c10) * b[1] + S(c20) * b[2]) / det;
    v6[4] = (S(c01) * b[0] + S(c11) * b[1] + S(c21) * b[2]) / det;
    v6[5] = (S(c02) * b[0] + S(c12) * b[1] + S(c22) * b[2]) / det;
  }
}
template <class S>
EXG_HD void inertia_apply(const double* I9, bool diag, bool kinematic, double mass, const S* v6, S* p6) {
  if (kinematic) {
#pragma unroll
    for (int c = 0; c < 6; ++c) p6[c] = v6[c];
    return;
  }
  S m = S(mass);
  p6[0] = v6[0] * m; p6[1] = v6[1] * m; p6[2] = v6[2] * m;
  if (diag) {
    p6[3] = S(I9[0]) * v6[3]; p6[4] = S(I9[4]) * v6[4]; p6[5] = S(I9[8]) * v6[5];
  } else {
    const S* w = v6 + 3;
    p6[3] = S(I9[0]) * w[0] + S(I9[1]) * w[1] + S(I9[2]) * w[2];
    p6[4] = S(I9[3]) * w[0] + S(I9[4]) * w[1] + S(I9[5]) * w[2];
    p6[5] = S(I9[6]) * w[0] + S(I9[7]) * w[1] + S(I9[8]) * w[2];
  }
}

EXG_HD void load_body(const BodyView& b, int i, double* pose8, double* mom6, double* I9) {
#pragma unroll
  for (int c = 0; c < 8; ++c) pose8[c] = b.pose[(size_t)c * b.n + i];
#pragma unroll
  for (int c = 0; c < 6; ++c) mom6[c] = b.mom[(size_t)c * b.n + i];
#pragma unroll
  for (int c = 0; c < 9; ++c) I9[c] = b.inertia[(size_t)c * b.n + i];
}

// position of the body origin
EXG_HD void body_position(const double* pose8, double* p3) {
  double zero[3] = {0.0, 0.0, 0.0}, pt[4];
  anchor_point(pose8, zero, pt);
  point_coords(pt, p3);
}

// world twist (lin, ang) from pose and body momentum
EXG_HD void world_velocity(const double* pose8, const double* mom6, const double* I9, bool diag, bool kin, double mass,
                           double* wv6) {
  double v6[6], vb[6], wb[6];
  inertia_inverse(I9, diag, kin, mass, mom6, v6);
  screw_from6(v6, vb);
  twist_transport(vb, pose8, wb);
  screw_to6(wb, wv6);
}

// UniformField (crates/newton/src/field.rs:29-47): the world force F = m a of a constant
// acceleration a (mass from the charge, 0 for kinematic bodies), added to the world wrench w6
// (force, torque about the world origin) as a force through the body's centre: (F, p x F).
EXG_HD void add_uniform_field(const double* a, const double4& pm, double* w6) {
  if (a[0] == 0.0 && a[1] == 0.0 && a[2] == 0.0) return;
  const double f[3] = {pm.w * a[0], pm.w * a[1], pm.w * a[2]};
  w6[0] += f[0];
  w6[1] += f[1];
  w6[2] += f[2];
  w6[3] += pm.y * f[2] - pm.z * f[1];
  w6[4] += pm.z * f[0] - pm.x * f[2];
  w6[5] += pm.x * f[1] - pm.y * f[0];
}

}  // namespace exg
