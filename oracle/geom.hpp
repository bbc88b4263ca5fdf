// ORACLE — test infrastructure only (CPU restatement the CUDA path is checked against).
//
// PGA3 rigid-body objects over the full multivector:
//   Motor (crates/clifford/src/pga3/motor.rs:109-283), Twist/Wrench = Screw<Contra/Co>
//   (crates/clifford/src/pga3/screw.rs:105-361), Point/Line (crates/clifford/src/pga3/objects.rs:20-175).
// Motor slot order = even blades in increasing bitmask order (motor.rs:119-147); a screw is
// the six grade-2 blades, written and read through the dual markup (mv.rs:619-705).
#pragma once
#include "pga3.hpp"
#include "scalar.hpp"

namespace oracle {

template <class T> using M = Mv<T>;

// ── Motor ────────────────────────────────────────────────────────────────
template <class T>
struct Motor {
  M<T> m;  // even grades only
  static Motor identity() { Motor r; r.m.c[0] = T(1.0); return r; }
  static Motor from_mv(const M<T>& x) { Motor r; r.m = x.even(); return r; }
  // motor.rs:119-133 / 136-147
  void to_components(T out[8]) const {
    int i = 0;
    for (int b = 0; b < DIM; ++b) if ((popc(unsigned(b)) & 1) == 0) out[i++] = m.c[b];
  }
  static Motor from_components(const T in[8]) {
    Motor r; int i = 0;
    for (int b = 0; b < DIM; ++b) if ((popc(unsigned(b)) & 1) == 0) r.m.c[b] = in[i++];
    return r;
  }
  // motor.rs:157-159: "first self, then rhs" = rhs * self
  Motor compose(const Motor& rhs) const { Motor r; r.m = rhs.m.gp(m); return r; }
  Motor inverse() const { Motor r; r.m = m.reverse(); return r; }
  M<T> conjugate_mv(const M<T>& x) const { return m.conjugate(x); }
  // motor.rs:199-217: closed-form screw exponential via Study numbers.
  static Motor exp_even(const M<T>& bs) {
    M<T> b2 = bs.gp(bs);
    T u = -b2.c[0];
    T p = b2.c[TOP];
    T cu = cos_sq(u), su = sinc_sq(u), du = dsinc_sq(u);
    M<T> i_mv = M<T>::basis(TOP);
    M<T> ib = i_mv.gp(bs);
    M<T> scalar_part = M<T>::scalar(cu) + i_mv.scale(p * T(0.5) * su);
    M<T> bivector_part = bs.scale(su) - ib.scale(p * du);
    Motor r; r.m = scalar_part + bivector_part; return r;
  }
  // motor.rs:228-242
  Motor normalized() const {
    T n2 = m.gp(m.reverse()).c[0];
    if (eff_zero(std_part(n2))) return *this;
    T inv = T(1.0) / s_sqrt(n2);
    Motor r; r.m = m.scale(inv); return r;
  }
  // motor.rs:244-250
  Motor rotation_part() const {
    Motor r;
    r.m.c[0] = m.c[0];
    V3<T> dir = read_dual(m, euclid_blade);
    write_dual(r.m, dir, euclid_blade);
    return r.normalized();
  }
};

// ── Screw (Twist = Contra, Wrench = Co) ─────────────────────────────────────
template <class T>
struct Screw {
  M<T> m;  // grade-2 only
  static Screw zero() { return Screw(); }
  static Screw from_mv(const M<T>& x) { Screw s; s.m = x.grade2(); return s; }
  // screw.rs:278-289 (twist) / 322-333 (wrench): linear/force -> radical blades,
  // angular/torque -> angular blades (Euclidean x computed sigma).
  static Screw make(const V3<T>& lin, const V3<T>& ang) {
    Screw s;
    write_dual(s.m, lin, radical_blade);
    write_dual(s.m, ang, angular_blade);
    return s;
  }
  V3<T> lin() const { return read_dual(m, radical_blade); }
  V3<T> ang() const { return read_dual(m, angular_blade); }
  void to6(T out[6]) const { V3<T> l = lin(), a = ang(); for (int i = 0; i < 3; ++i) { out[i] = l[i]; out[3 + i] = a[i]; } }
  static Screw from6(const T in[6]) { return make(V3<T>(in[0], in[1], in[2]), V3<T>(in[3], in[4], in[5])); }
  Screw operator+(const Screw& o) const { Screw s; s.m = m + o.m; return s; }
  Screw operator-(const Screw& o) const { Screw s; s.m = m - o.m; return s; }
  Screw operator-() const { Screw s; s.m = -m; return s; }
  Screw scale(const T& k) const { Screw s; s.m = m.scale(k); return s; }
  // screw.rs:94-99 (Contra) and 100-105 (Co)
  Screw transport_contra(const Motor<T>& mo) const { return from_mv(mo.m.conjugate(m)); }
  Screw transport_co(const Motor<T>& mo) const { return from_mv(mo.m.conjugate(m.dual()).undual()); }
};
template <class T> using Twist = Screw<T>;
template <class T> using Wrench = Screw<T>;

// screw.rs:297-301: exp(dt) = Motor::exp(t * dt/2)
template <class T> inline Motor<T> twist_exp(const Twist<T>& t, const T& dt) {
  return Motor<T>::exp_even(t.scale(dt * T(0.5)).m);
}
template <class T> inline Motor<T> motor_exp(const Twist<T>& t) { return Motor<T>::exp_even(t.m); }

// screw.rs:355-361: pairing <w ^ dual(t)>_I
template <class T> inline T power(const Wrench<T>& w, const Twist<T>& t) { return w.m.wedge(t.m.dual()).c[TOP]; }
// screw.rs:347-357: the coadjoint action, one half of undual([t, dual(w)])
template <class T> inline Wrench<T> coad_bracket(const Wrench<T>& w, const Twist<T>& t) {
  M<T> raw = t.m.commutator(w.m.dual()).undual();
  return Wrench<T>::from_mv(raw).scale(T(0.5));
}

// ── Points and lines ───────────────────────────────────────────────────────
template <class T>
struct Point {
  M<T> m;
  static Point at(const V3<T>& v) {  // mv.rs:582-593
    Point p; p.m.c[I3] = T(1.0);
    write_dual(p.m, v, point_blade);
    return p;
  }
  V3<T> coords() const {  // mv.rs:566-580: projective normalisation by the weight
    T winv = T(1.0) / m.c[I3];
    V3<T> raw = read_dual(m, point_blade);
    return raw.scale(winv);
  }
  M<T> join(const Point& o) const { return m.meet(o.m); }  // objects.rs:42-45
};
// Direction readers of a line (mv.rs:640-650).
template <class T> inline V3<T> line_direction(const M<T>& l) { return read_dual(l, euclid_blade); }
template <class T> inline V3<T> line_moment(const M<T>& l) { return read_dual(l, radical_blade); }
template <class T> inline T line_weight_norm(const M<T>& l) { return s_sqrt(l.norm_squared()); }
// objects.rs:120-122 / mv.rs:436-438
template <class T> inline T soft_weight_norm(const M<T>& l, const T& eps) { return s_sqrt(l.norm_squared() + eps * eps); }
// screw.rs:337-339: a wrench along a line of action
template <class T> inline Wrench<T> from_line(const M<T>& l) { return Wrench<T>::from_mv(l.dual()); }
// screw.rs:310-314: v = one half of [T, P], read as a direction
template <class T> inline V3<T> velocity_at(const Twist<T>& t, const Point<T>& p) {
  M<T> comm = t.m.commutator(p.m).scale(T(0.5));
  return read_dual(comm, point_blade);
}
// joints/src/lib.rs:258-263
template <class T> inline Point<T> anchor_point(const Motor<T>& pose, const V3<T>& local) {
  Point<T> p; p.m = pose.m.conjugate(Point<T>::at(local).m); return p;
}

}  // namespace oracle
