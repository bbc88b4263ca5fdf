// Rigid-motion operations used by the force laws and the integrators, on the narrow
// carriers of pga3.cuh. Each one restates an operation of the reference's PGA3 facade:
// screw exponential (crates/clifford/src/pga3/motor.rs:199-217), versor normalisation and
// rotational part (motor.rs:228-250), join of points (pga3/objects.rs:42-45), line norms
// (objects.rs:103-122), wrench of a line (screw.rs:337-339), power pairing (screw.rs:355-361),
// velocity of a twist at a point (screw.rs:310-314) and the coadjoint bracket (screw.rs:347-357).
#pragma once
#include "scalar.cuh"

namespace exg {

// Motor = exp(B) for a bivector B via the Study numbers of B*B.
template <class S> EXG_HD void motor_exp_biv(const S* b, S* m) {
  S b2[2];
  gp<BIV, BIV, SCL_PSC>(b, b, b2);
  S u = -b2[0], p = b2[1];
  S cu = cos_sq(u), su = sinc_sq(u), du = dsinc_sq(u);
  S one[1] = {S(1.0)};
  S ib[6];
  gp<PSC, BIV, BIV>(one, b, ib);
  m[0] = cu;
  m[7] = p * S(0.5) * su;
  static_for<0, 6>([&](auto i) {
    constexpr int s = slot_of(EVEN, BIV[i]);
    m[s] = b[i] * su - ib[i] * (p * du);
  });
}
// Twist::exp(dt) = exp(t * dt / 2) (screw.rs:297-301)
template <class S> EXG_HD void twist_exp(const S* t, const S& dt, S* m) {
  S h = dt * S(0.5);
  S b[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) b[i] = t[i] * h;
  motor_exp_biv(b, m);
}
template <class S> EXG_HD S even_norm2(const S* m) {
  S r[8], n[1];
  reverse<EVEN>(m, r);
  gp<EVEN, EVEN, SCL>(m, r, n);
  return n[0];
}
template <class S> EXG_HD void motor_normalized(const S* m, S* out) {
  S n2 = even_norm2(m);
  if (eff_zero(n2)) {
#pragma unroll
    for (int i = 0; i < 8; ++i) out[i] = m[i];
    return;
  }
  S inv = S(1.0) / s_sqrt(n2);
#pragma unroll
  for (int i = 0; i < 8; ++i) out[i] = m[i] * inv;
}
// scalar + Euclidean bivector, normalised
template <class S> EXG_HD void motor_rotation_part(const S* m, S* out) {
  S r[8];
  r[0] = m[0];
  static_for<1, 8>([&](auto i) {
    constexpr int bl = EVEN[i];
    if constexpr ((bl & kZeroMask) == 0 && cpopc(bl) == 2) r[i] = m[i]; else r[i] = S(0.0);
  });
  motor_normalized(r, out);
}

// Join of two points: undual(dual(P) ^ dual(Q)) — the grade-2 part of the product of the
// two dual vectors is their wedge.
template <class S> EXG_HD void point_join(const S* p, const S* q, S* line) {
  S dp[4], dq[4], w[6];
  dual_map<PNT, VEC, false>(p, dp);
  dual_map<PNT, VEC, false>(q, dq);
  gp<VEC, VEC, BIV>(dp, dq, w);
  dual_map<BIV, BIV, true>(w, line);
}
template <class S> EXG_HD S biv_norm2(const S* l) {
  S r[6], n[1];
  reverse<BIV>(l, r);
  gp<BIV, BIV, SCL>(l, r, n);
  return n[0];
}
template <class S> EXG_HD S soft_weight_norm(const S* l, const S& eps) { return s_sqrt(biv_norm2(l) + eps * eps); }
template <class S> EXG_HD void wrench_from_line(const S* l, S* w) { dual_map<BIV, BIV, false>(l, w); }
// <w ^ dual(t)>_I
template <class S> EXG_HD S screw_power(const S* w, const S* t) {
  S dt[6], p[1];
  dual_map<BIV, BIV, false>(t, dt);
  gp<BIV, BIV, PSC>(w, dt, p);
  return p[0];
}
// linear velocity of twist t at point p: one half of the point part of (t p - p t)
template <class S> EXG_HD void velocity_at(const S* t, const S* p, S* v) {
  S tp[4], pt[4], c[4];
  gp<BIV, PNT, PNT>(t, p, tp);
  gp<PNT, BIV, PNT>(p, t, pt);
#pragma unroll
  for (int i = 0; i < 4; ++i) c[i] = (tp[i] - pt[i]) * S(0.5);
  point_read<PNT>(c, v);
}
// one half of undual(t dual(w) - dual(w) t)
template <class S> EXG_HD void coad_bracket(const S* w, const S* t, S* out) {
  S dw[6], a[6], b[6], c[6];
  dual_map<BIV, BIV, false>(w, dw);
  gp<BIV, BIV, BIV>(t, dw, a);
  gp<BIV, BIV, BIV>(dw, t, b);
#pragma unroll
  for (int i = 0; i < 6; ++i) c[i] = a[i] - b[i];
  dual_map<BIV, BIV, true>(c, out);
#pragma unroll
  for (int i = 0; i < 6; ++i) out[i] = out[i] * S(0.5);
}

// physical (lin, ang) helpers
template <class S> EXG_HD void screw_from6(const S* x6, S* biv) { screw_from_phys(x6, x6 + 3, biv); }
template <class S> EXG_HD void screw_to6(const S* biv, S* x6) { screw_to_phys(biv, x6, x6 + 3); }

}  // namespace exg
