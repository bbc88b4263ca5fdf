// Device algebra for PGA3 = Cl(3,0,1): compile-time sparse geometric products on narrow
// carriers, templated on the scalar (double, float, Dual<N, R>).
//
// Conventions are the reference's (crates/clifford/src/algebra/mod.rs:84-140,
// algebra/markup.rs:13-100): the generator chain puts e1, e2, e3 on bits 0..2 and the
// degenerate e0 on bit 3; a blade is a bitmask, its product sign is the merge-permutation
// parity times the metric; dual is the complement with b ^ dual(b) = +I. Every table below
// is evaluated by the compiler from those laws, and every product is unrolled into straight
// line code at compile time: a blade pair whose sign is zero, or whose result falls outside
// the requested output carrier, emits no instruction.
//
// Carriers (blade lists, increasing bitmask):
//   EVEN  {0,3,5,6,9,10,12,15}  motor (crates/clifford/src/pga3/motor.rs:119-147)
//   BIV   {3,5,6,9,10,12}        screw: twist / wrench / line (pga3/screw.rs:105-130)
//   PNT   {7,11,13,14}           point (weight on 7)
//   VEC   {1,2,4,8}              plane / dual of a point
//   ODD   {1,2,4,7,8,11,13,14}   intermediate of a point sandwich
#pragma once
#include <cstdint>
#include <type_traits>
#include <utility>

#if defined(__CUDACC__)
#define EXG_HD __host__ __device__ __forceinline__
#else
#define EXG_HD inline
#endif

namespace exg {

// ── the sign law, evaluated at compile time ──────────────────────────────────
constexpr int kZeroMask = 0b1000;
constexpr int kTop = 15;
constexpr int kI3 = kTop & ~kZeroMask;

constexpr int cpopc(int x) { int c = 0; while (x) { c += x & 1; x >>= 1; } return c; }

struct CProd { int sign; int mask; };
constexpr CProd cprod(int a, int b) {
  if ((a & b) & kZeroMask) return {0, 0};
  int swaps = 0;
  for (int aa = a >> 1; aa; aa >>= 1) swaps += cpopc(aa & b);
  return {(swaps & 1) ? -1 : 1, a ^ b};
}
constexpr int ccomplement_sign(int a, int b) {
  int inv = 0;
  for (int bi = 0; bi < 4; ++bi)
    if ((a >> bi) & 1) inv += cpopc(b & ((1 << bi) - 1));
  return (inv & 1) ? -1 : 1;
}
constexpr int caxis(int i) {
  int e = kI3;
  for (;;) {
    int low = e & -e;
    if (i == 0) return low;
    e ^= low;
    --i;
  }
}
struct CMark { int mask; int sign; };
constexpr CMark euclid_mark(int i) { int v = caxis(i); int c = kI3 ^ v; return {c, ccomplement_sign(v, c)}; }
constexpr CMark radical_mark(int i) { CProd p = cprod(kZeroMask, caxis(i)); return {p.mask, p.sign}; }
constexpr CMark point_mark(int i) {
  CMark e = euclid_mark(i);
  CProd p = cprod(kZeroMask, e.mask);
  return {p.mask, e.sign * p.sign};
}
// The angular embedding sign is solved from velocity = omega x r read through the point
// markup and through the Euclidean cross product (the reference derives it the same way).
constexpr int angular_sigma() {
  CProd w = cprod(caxis(2), caxis(0));
  CMark e1 = euclid_mark(1), b = euclid_mark(2), p = point_mark(0), d = point_mark(1);
  int hs = (cprod(b.mask, p.mask).sign - cprod(p.mask, b.mask).sign) / 2;
  return e1.sign * w.sign * d.sign * hs * b.sign * p.sign;
}
constexpr CMark angular_mark(int i) { CMark m = euclid_mark(i); return {m.mask, m.sign * angular_sigma()}; }

template <int N> struct Blades { int b[N]; constexpr int operator[](int i) const { return b[i]; } static constexpr int size = N; };
constexpr Blades<8> EVEN{{0, 3, 5, 6, 9, 10, 12, 15}};
constexpr Blades<6> BIV{{3, 5, 6, 9, 10, 12}};
constexpr Blades<4> PNT{{7, 11, 13, 14}};
constexpr Blades<4> VEC{{1, 2, 4, 8}};
constexpr Blades<8> ODD{{1, 2, 4, 7, 8, 11, 13, 14}};
constexpr Blades<1> SCL{{0}};
constexpr Blades<1> PSC{{15}};
constexpr Blades<2> SCL_PSC{{0, 15}};

template <int N> constexpr int slot_of(const Blades<N>& l, int mask) {
  for (int i = 0; i < N; ++i) if (l.b[i] == mask) return i;
  return -1;
}
static_assert(angular_sigma() == 1 || angular_sigma() == -1, "sign law");

// ── compile-time loops ─────────────────────────────────────────────────────
template <int I, int N, class F> EXG_HD void static_for(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

// Is (i, j) the first blade pair contributing to output slot o?  Lets a product write its
// first term instead of adding it to zero.
template <const auto& LA, const auto& LB, const auto& LO>
constexpr int first_pair(int o) {
  for (int i = 0; i < LA.size; ++i)
    for (int j = 0; j < LB.size; ++j) {
      CProd p = cprod(LA[i], LB[j]);
      if (p.sign != 0 && slot_of(LO, p.mask) == o) return i * LB.size + j;
    }
  return -1;
}

// out = project_LO(a * b), a on carrier LA, b on carrier LB.
template <const auto& LA, const auto& LB, const auto& LO, class S>
EXG_HD void gp(const S* a, const S* b, S* out) {
  static_for<0, LO.size>([&](auto o) {
    if constexpr (first_pair<LA, LB, LO>(o) < 0) out[o] = S(0.0);
  });
  static_for<0, LA.size * LB.size>([&](auto k) {
    constexpr int i = k / LB.size, j = k % LB.size;
    constexpr CProd p = cprod(LA[i], LB[j]);
    if constexpr (p.sign != 0) {
      constexpr int o = slot_of(LO, p.mask);
      if constexpr (o >= 0) {
        constexpr bool first = first_pair<LA, LB, LO>(o) == k;
        if constexpr (first) {
          if constexpr (p.sign > 0) out[o] = a[i] * b[j]; else out[o] = -(a[i] * b[j]);
        } else {
          if constexpr (p.sign > 0) out[o] = out[o] + a[i] * b[j]; else out[o] = out[o] - a[i] * b[j];
        }
      }
    }
  });
}

// dual / undual of a carrier onto the complementary carrier (mv.rs:220-252)
template <const auto& LI, const auto& LO, bool Undual, class S>
EXG_HD void dual_map(const S* a, S* out) {
  static_for<0, LI.size>([&](auto i) {
    constexpr int s = LI[i];
    constexpr int comp = kTop ^ s;
    constexpr int o = slot_of(LO, comp);
    static_assert(o >= 0, "dual lands outside the output carrier");
    constexpr int sg = Undual ? ccomplement_sign(comp, s) : ccomplement_sign(s, comp);
    if constexpr (sg > 0) out[o] = a[i]; else out[o] = -a[i];
  });
}

// reverse on a carrier: sign (-1)^(g(g-1)/2)
template <const auto& L, class S>
EXG_HD void reverse(const S* a, S* out) {
  static_for<0, L.size>([&](auto i) {
    constexpr int g = cpopc(L[i]);
    if constexpr (((g * (g - 1)) / 2) & 1) out[i] = -a[i]; else out[i] = a[i];
  });
}

// ── physical markup on the screw carrier ────────────────────────────────────
// A screw is stored in BIV blade order. Twist/wrench (lin|force xyz, ang|torque xyz) are
// written through the radical and angular markups (mv.rs:690-705).
template <class S> EXG_HD void screw_from_phys(const S* lin, const S* ang, S* biv) {
  static_for<0, 3>([&](auto i) {
    constexpr CMark r = radical_mark(i);
    constexpr CMark a = angular_mark(i);
    constexpr int sr = slot_of(BIV, r.mask), sa = slot_of(BIV, a.mask);
    if constexpr (r.sign > 0) biv[sr] = lin[i]; else biv[sr] = -lin[i];
    if constexpr (a.sign > 0) biv[sa] = ang[i]; else biv[sa] = -ang[i];
  });
}
template <class S> EXG_HD void screw_to_phys(const S* biv, S* lin, S* ang) {
  static_for<0, 3>([&](auto i) {
    constexpr CMark r = radical_mark(i);
    constexpr CMark a = angular_mark(i);
    constexpr int sr = slot_of(BIV, r.mask), sa = slot_of(BIV, a.mask);
    if constexpr (r.sign > 0) lin[i] = biv[sr]; else lin[i] = -biv[sr];
    if constexpr (a.sign > 0) ang[i] = biv[sa]; else ang[i] = -biv[sa];
  });
}
// A line's direction (Euclidean blades) and moment (radical blades) (mv.rs:640-650).
template <class S> EXG_HD void line_direction(const S* biv, S* dir) {
  static_for<0, 3>([&](auto i) {
    constexpr CMark e = euclid_mark(i);
    constexpr int s = slot_of(BIV, e.mask);
    if constexpr (e.sign > 0) dir[i] = biv[s]; else dir[i] = -biv[s];
  });
}
// Point (weight 1) at coordinates v, and back with projective normalisation (mv.rs:566-593).
template <class S> EXG_HD void point_make(const S* v, S* p) {
  p[slot_of(PNT, kI3)] = S(1.0);
  static_for<0, 3>([&](auto i) {
    constexpr CMark m = point_mark(i);
    constexpr int s = slot_of(PNT, m.mask);
    if constexpr (m.sign > 0) p[s] = v[i]; else p[s] = -v[i];
  });
}
template <const auto& L, class S> EXG_HD void point_read(const S* p, S* v) {  // no weight division
  static_for<0, 3>([&](auto i) {
    constexpr CMark m = point_mark(i);
    constexpr int s = slot_of(L, m.mask);
    if constexpr (m.sign > 0) v[i] = p[s]; else v[i] = -p[s];
  });
}
template <class S> EXG_HD void point_coords(const S* p, S* v) {
  S winv = S(1.0) / p[slot_of(PNT, kI3)];
  point_read<PNT>(p, v);
  v[0] = v[0] * winv; v[1] = v[1] * winv; v[2] = v[2] * winv;
}

// ── motors ──────────────────────────────────────────────────────────────────
// compose(a, b): "first a, then b" = b * a (motor.rs:157-159)
template <class S> EXG_HD void motor_compose(const S* a, const S* b, S* out) { gp<EVEN, EVEN, EVEN>(b, a, out); }
template <class S> EXG_HD void motor_reverse(const S* a, S* out) { reverse<EVEN>(a, out); }

// Ad: M t M~ on a bivector (screw.rs:94-99)
template <class S> EXG_HD void biv_conjugate(const S* m, const S* t, S* out) {
  S mt[8], mr[8];
  gp<EVEN, BIV, EVEN>(m, t, mt);
  reverse<EVEN>(m, mr);
  gp<EVEN, EVEN, BIV>(mt, mr, out);
}
// twist transport (Contra) and wrench transport (Co = undual(M dual(w) M~)) (screw.rs:94-105)
template <class S> EXG_HD void twist_transport(const S* t, const S* m, S* out) { biv_conjugate(m, t, out); }
template <class S> EXG_HD void wrench_transport(const S* w, const S* m, S* out) {
  S d[6], c[6];
  dual_map<BIV, BIV, false>(w, d);
  biv_conjugate(m, d, c);
  dual_map<BIV, BIV, true>(c, out);
}
// point sandwich M P M~ (the weight stays on the point carrier)
template <class S> EXG_HD void point_conjugate(const S* m, const S* p, S* out) {
  S mp[8], mr[8];
  gp<EVEN, PNT, ODD>(m, p, mp);
  reverse<EVEN>(m, mr);
  gp<ODD, EVEN, PNT>(mp, mr, out);
}
// world point of a local anchor (joints/src/lib.rs:258-263)
template <class S> EXG_HD void anchor_point(const S* m, const S* local, S* p) {
  S q[4];
  point_make(local, q);
  point_conjugate(m, q, p);
}

// Study-form transcendentals with the representation seams of the reference
// (crates/peano/src/scalar.rs:67-131). The seam threshold is that of the carrier's standard
// part: 1e-9 for double, 1e-5 for float (crates/peano/src/support.rs:39-49).
template <class S> struct ScalarTraits;
template <> struct ScalarTraits<double> {
  using Real = double;
  static EXG_HD double std_part(double x) { return x; }
  static EXG_HD bool eff_zero(double x) { return (x < 0 ? -x : x) < 1e-9; }
};
template <> struct ScalarTraits<float> {
  using Real = float;
  static EXG_HD float std_part(float x) { return x; }
  static EXG_HD bool eff_zero(float x) { return (x < 0 ? -x : x) < 1e-5f; }
};

}  // namespace exg
