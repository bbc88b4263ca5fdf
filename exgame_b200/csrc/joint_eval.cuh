// Per-joint evaluation routines shared by the joint kernels.
//
// Plain:    the 12 wrench components [force a, torque a, force b, torque b] at (pose, twist)
//           (crates/newton/build.rs:938-973).
// Jacobian: value + partials w.r.t. 24 axes — pose A, pose B (retraction exp(delta) * pose,
//           unit Motor::exp, no half), world twist A, world twist B, each lin xyz then ang xyz
//           (crates/newton/build.rs:673-768, crates/clifford/src/pga3/ad.rs:119-150).
//           The 24 axes are evaluated as four 6-axis dual slices; slice s seeds axes
//           6s..6s+5. With the pose seed's value at zero, exp(delta) = 1 + delta exactly to
//           first order (the Study forms take their Taylor arm at u = 0), so the seeded pose
//           is (1 + delta) * pose.
// The wrench on b is the negation of the wrench on a for every law, so only a is evaluated.
#pragma once
#include "laws.cuh"

namespace exg {

// poses: 8 motor components in slot order; twists: 6 physical components (lin, ang).
template <class R>
EXG_HD void joint_plain(int law, const double* prm, const R* pose_a, const R* pose_b, const R* vel_a, const R* vel_b, double dt,
                        double warp, R* out12) {
  R ta[6], tb[6], wa[6];
  screw_from6(vel_a, ta);
  screw_from6(vel_b, tb);
  law_wrench(law, prm, pose_a, pose_b, ta, tb, dt, warp, wa);
  R w6[6];
  screw_to6(wa, w6);
#pragma unroll
  for (int i = 0; i < 6; ++i) { out12[i] = w6[i]; out12[6 + i] = -w6[i]; }
}

// One slice: value[6] of the wrench on a and d[6][6] = d(wrench on a component r)/d(axis 6s+c),
// stored d[r*6 + c]. With N = 3 one call evaluates half a slice — the axes 6s + 3h .. 6s + 3h + 2
// (h = half) — and fills columns 3h .. 3h + 2 of d (value6 as well); each derivative column is
// computed by the same dual operations whatever N is, so two halves give the full slice's values
// bit for bit with about half the live state per thread.
// KIND = 0 / 1 promises a pose / twist slice at compile time (-1: decided by `slice`).
template <class R, int N = 6, int KIND = -1>
EXG_HD void joint_jacobian_part(int law, const double* prm, const R* pose_a, const R* pose_b, const R* vel_a,
                                const R* vel_b, double dt, double warp, int slice, int half, R* value6, R* d36) {
  static_assert(N == 6 || N == 3, "a slice is evaluated whole or in halves");
  const int c0 = N == 6 ? 0 : 3 * half;
  if (law == LAW_TORSIONAL) {
    // The couple -k (w_a - w_b) depends on the angular velocities only, linearly: its Jacobian is
    // -k I (velocity A) and +k I (velocity B) on the torque rows, zero elsewhere — exactly what the
    // dual evaluation produces, without the dual arithmetic.
    R ta[6], tb[6], wa[6], w6[6];
    screw_from6(vel_a, ta);
    screw_from6(vel_b, tb);
    law_torsional(prm, ta, tb, warp, wa);
    screw_to6(wa, w6);
#pragma unroll
    for (int r = 0; r < 6; ++r) value6[r] = w6[r];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = 0; c < N; ++c) d36[r * 6 + c0 + c] = R(0.0);
    if (slice >= 2) {
      R k = -R(prm[0] / (warp * warp));
      R g = slice == 2 ? k : -k;
#pragma unroll
      for (int r = 3; r < 6; ++r)
        if (r >= c0 && r < c0 + N) d36[r * 6 + r] = g;
    }
    return;
  }
  using D = Dual<N, R>;
  // the wrench's value and its N partial columns into value6 / d36
  auto emit = [&](const D* wa) {
    D w6[6];
    screw_to6(wa, w6);
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      value6[r] = w6[r].v;
#pragma unroll
      for (int c = 0; c < N; ++c) d36[r * 6 + c0 + c] = w6[r].g[c];
    }
  };
  // Each branch ends in its own emit: the two paths share no arrays after the branch, which
  // keeps them in registers.
  if (KIND == 0 || (KIND < 0 && slice < 2)) {
    D ma[8], mb[8], va[6], vb[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) { va[i] = D(0.0); va[i].v = vel_a[i]; vb[i] = D(0.0); vb[i].v = vel_b[i]; }
#pragma unroll
    for (int i = 0; i < 8; ++i) { ma[i] = D(0.0); ma[i].v = pose_a[i]; mb[i] = D(0.0); mb[i].v = pose_b[i]; }
    // pose seed: (1 + delta) * base with delta = Twist(seed lin, seed ang), value 0
    D seed6[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      seed6[i] = D(0.0);
#pragma unroll
      for (int c = 0; c < N; ++c) seed6[i].g[c] = (i == c0 + c) ? R(1) : R(0);  // static register index
    }
    D delta[6], one_delta[8];
    screw_from6(seed6, delta);
    one_delta[0] = D(1.0);
    one_delta[7] = D(0.0);
    static_for<0, 6>([&](auto i) { one_delta[slot_of(EVEN, BIV[i])] = delta[i]; });
    // the seeded pose (a or b) by selects, so the arrays stay in registers
    const bool on_a = slice == 0;
    D base[8], moved[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) base[i] = on_a ? ma[i] : mb[i];
    gp<EVEN, EVEN, EVEN>(one_delta, base, moved);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      ma[i] = on_a ? moved[i] : ma[i];
      mb[i] = on_a ? mb[i] : moved[i];
    }
    D ta[6], tb[6], wa[6];
    screw_from6(va, ta);
    screw_from6(vb, tb);
    law_wrench<D, D>(law, prm, ma, mb, ta, tb, dt, warp, wa);
    emit(wa);
  } else {
    // twist seed: the poses carry no partials, so the laws' pose chains run plain
    D va[6], vb[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) { va[i] = D(0.0); va[i].v = vel_a[i]; vb[i] = D(0.0); vb[i].v = vel_b[i]; }
    const bool on_a = slice == 2;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int c = 0; c < N; ++c) {
        const R one = (i == c0 + c) ? R(1) : R(0);  // static register index
        va[i].g[c] = on_a ? one : R(0);
        vb[i].g[c] = on_a ? R(0) : one;
      }
    D ta[6], tb[6], wa[6];
    screw_from6(va, ta);
    screw_from6(vb, tb);
    law_wrench<D, R>(law, prm, pose_a, pose_b, ta, tb, dt, warp, wa);
    emit(wa);
  }
}

template <class R>
EXG_HD void joint_jacobian_slice(int law, const double* prm, const R* pose_a, const R* pose_b, const R* vel_a,
                                 const R* vel_b, double dt, double warp, int slice, R* value6, R* d36) {
  joint_jacobian_part<R, 6>(law, prm, pose_a, pose_b, vel_a, vel_b, dt, warp, slice, 0, value6, d36);
}

}  // namespace exg
