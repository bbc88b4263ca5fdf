// ORACLE — test infrastructure only. This file is the CPU restatement that the
// CUDA path is checked against; nothing in the shipped library includes it.
//
// Projective geometric algebra Cl(3,0,1) restated from the reference's sign law:
//   * generator chain Gen<0, Gen<1, Gen<1, Gen<1, Nil>>>>: the innermost generator
//     is bit 0, e0 (square 0) is the outermost one, bit 3
//     (crates/clifford/src/algebra/mod.rs:84-90);
//   * blade product sign = parity of the merge permutation x metric, a degenerate
//     shared generator annihilates (crates/clifford/src/algebra/mod.rs:100-117);
//   * dual = complement with b ^ dual(b) = +I (crates/clifford/src/algebra/mod.rs:119-140,
//     crates/clifford/src/algebra/mv.rs:220-232), undual with the argument order swapped
//     (mv.rs:240-252);
//   * the physical markup (axis, euclid, radical, point, angular blades) is COMPUTED from
//     those two laws (crates/clifford/src/algebra/markup.rs:13-100), never tabulated.
// The multivector is a plain 16-slot array indexed by blade bitmask; every product is a
// runtime loop over blade pairs, like the reference's `graded_gp` (mv.rs:190-212). The
// narrow carriers (Motor: 8 even slots, Screw: 6 grade-2 slots) are views over it.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>

namespace oracle {

constexpr int NGEN = 4;
constexpr int DIM = 16;
constexpr int TOP = DIM - 1;
constexpr int ZERO_MASK = 0b1000;  // e0
constexpr int NEG_MASK = 0;
constexpr int I3 = TOP & ~ZERO_MASK;  // Euclidean pseudoscalar e123 = 0b0111

inline int popc(unsigned x) { return __builtin_popcount(x); }

struct BladeProd { int sign; int mask; };

// crates/clifford/src/algebra/mod.rs:100-117
inline BladeProd blade_prod(int a, int b) {
  int shared = a & b;
  if (shared & ZERO_MASK) return {0, 0};
  int neg = popc(unsigned(shared & NEG_MASK)) & 1;
  int swaps = 0;
  int aa = a >> 1;
  while (aa) { swaps += popc(unsigned(aa & b)); aa >>= 1; }
  return {((swaps + neg) & 1) ? -1 : 1, a ^ b};
}

constexpr int DUAL_ORIENTATION = 1;
// crates/clifford/src/algebra/mod.rs:125-140
inline int complement_sign(int a, int b) {
  int inv = 0;
  for (int bi = 0; bi < 8; ++bi)
    if ((a >> bi) & 1) inv += popc(unsigned(b & ((1 << bi) - 1)));
  return (inv % 2 == 0) ? DUAL_ORIENTATION : -DUAL_ORIENTATION;
}

struct MaskSign { int mask; int sign; };

// crates/clifford/src/algebra/markup.rs:13-26
inline int axis_vec(int i) {
  int e = I3;
  for (;;) {
    int low = e & -e;
    if (i == 0) return low;
    e ^= low;
    --i;
  }
}
// markup.rs:30-35
inline MaskSign euclid_blade(int i) {
  int v = axis_vec(i);
  int comp = I3 ^ v;
  return {comp, complement_sign(v, comp)};
}
// markup.rs:39-43
inline MaskSign radical_blade(int i) {
  int v = axis_vec(i);
  BladeProd p = blade_prod(ZERO_MASK, v);
  return {p.mask, p.sign};
}
// markup.rs:46-50
inline MaskSign point_blade(int i) {
  MaskSign ec = euclid_blade(i);
  BladeProd p = blade_prod(ZERO_MASK, ec.mask);
  return {p.mask, ec.sign * p.sign};
}
// markup.rs:66-82: the embedding sign of the angular generator, solved from
// velocity = omega x r read through two independently derived channels.
inline int angular_embed_sign() {
  int vz = axis_vec(2), vx = axis_vec(0);
  BladeProd w = blade_prod(vz, vx);
  MaskSign e1 = euclid_blade(1);
  MaskSign b = euclid_blade(2);
  MaskSign p = point_blade(0);
  MaskSign d = point_blade(1);
  BladeProd s1 = blade_prod(b.mask, p.mask);
  BladeProd s2 = blade_prod(p.mask, b.mask);
  int hs = (s1.sign - s2.sign) / 2;
  (void)w.mask; (void)e1.mask; (void)d.mask;
  return e1.sign * w.sign * d.sign * hs * b.sign * p.sign;
}
// markup.rs:86-89
inline MaskSign angular_blade(int i) {
  MaskSign m = euclid_blade(i);
  return {m.mask, m.sign * angular_embed_sign()};
}

// Precomputed product table (sign, result mask) for every blade pair.
struct GpTable {
  signed char sign[DIM][DIM];
  unsigned char mask[DIM][DIM];
  GpTable() {
    for (int a = 0; a < DIM; ++a)
      for (int b = 0; b < DIM; ++b) {
        BladeProd p = blade_prod(a, b);
        sign[a][b] = (signed char)p.sign;
        mask[a][b] = (unsigned char)p.mask;
      }
  }
};
inline const GpTable& gp_table() { static GpTable t; return t; }

template <class T> inline bool structurally_zero(const T& x);
template <> inline bool structurally_zero<double>(const double& x) { return x == 0.0; }
template <> inline bool structurally_zero<float>(const float& x) { return x == 0.0f; }

// ── Full multivector ──────────────────────────────────────────────────────
template <class T>
struct Mv {
  std::array<T, DIM> c;
  Mv() { for (auto& x : c) x = T(0.0); }
  static Mv scalar(T s) { Mv m; m.c[0] = s; return m; }
  static Mv basis(int blade) { Mv m; m.c[blade] = T(1.0); return m; }
  T get(int b) const { return c[b]; }
  Mv operator+(const Mv& o) const { Mv r; for (int i = 0; i < DIM; ++i) r.c[i] = c[i] + o.c[i]; return r; }
  Mv operator-(const Mv& o) const { Mv r; for (int i = 0; i < DIM; ++i) r.c[i] = c[i] - o.c[i]; return r; }
  Mv operator-() const { Mv r; for (int i = 0; i < DIM; ++i) r.c[i] = -c[i]; return r; }
  Mv scale(const T& s) const { Mv r; for (int i = 0; i < DIM; ++i) r.c[i] = c[i] * s; return r; }

  // Geometric product (crates/clifford/src/algebra/mv.rs:262-266): sum over blade pairs.
  Mv gp(const Mv& o) const {
    const GpTable& t = gp_table();
    Mv r;
    for (int a = 0; a < DIM; ++a) {
      if (structurally_zero(c[a])) continue;
      for (int b = 0; b < DIM; ++b) {
        int s = t.sign[a][b];
        if (s == 0 || structurally_zero(o.c[b])) continue;
        T term = c[a] * o.c[b];
        int m = t.mask[a][b];
        if (s < 0) r.c[m] = r.c[m] - term; else r.c[m] = r.c[m] + term;
      }
    }
    return r;
  }
  // Grade-filtered products (mv.rs:190-218).
  Mv graded(const Mv& o, bool wedge) const {
    const GpTable& t = gp_table();
    Mv r;
    for (int a = 0; a < DIM; ++a) {
      if (structurally_zero(c[a])) continue;
      int ga = popc(unsigned(a));
      for (int b = 0; b < DIM; ++b) {
        int s = t.sign[a][b];
        if (s == 0 || structurally_zero(o.c[b])) continue;
        int gb = popc(unsigned(b));
        int m = t.mask[a][b];
        int want = wedge ? ga + gb : (ga > gb ? ga - gb : gb - ga);
        if (popc(unsigned(m)) != want) continue;
        T term = c[a] * o.c[b];
        if (s < 0) r.c[m] = r.c[m] - term; else r.c[m] = r.c[m] + term;
      }
    }
    return r;
  }
  Mv wedge(const Mv& o) const { return graded(o, true); }
  Mv dot(const Mv& o) const { return graded(o, false); }
  // Involutions (mv.rs:150-170).
  Mv reverse() const {
    Mv r;
    for (int b = 0; b < DIM; ++b) {
      unsigned g = popc(unsigned(b));
      bool flip = ((g * (g - 1)) / 2) & 1;
      r.c[b] = flip ? -c[b] : c[b];
    }
    return r;
  }
  // mv.rs:220-232
  Mv dual() const {
    Mv r;
    for (int s = 0; s < DIM; ++s) {
      int comp = TOP ^ s;
      r.c[comp] = r.c[comp] + (complement_sign(s, comp) < 0 ? -c[s] : c[s]);
    }
    return r;
  }
  // mv.rs:240-252
  Mv undual() const {
    Mv r;
    for (int s = 0; s < DIM; ++s) {
      int comp = TOP ^ s;
      r.c[comp] = r.c[comp] + (complement_sign(comp, s) < 0 ? -c[s] : c[s]);
    }
    return r;
  }
  Mv meet(const Mv& o) const { return dual().wedge(o.dual()).undual(); }
  Mv commutator(const Mv& o) const { return gp(o) - o.gp(*this); }
  Mv conjugate(const Mv& x) const { return gp(x).gp(reverse()); }
  T norm_squared() const { return gp(reverse()).c[0]; }
  Mv grade2() const {
    Mv r;
    for (int b = 0; b < DIM; ++b) if (popc(unsigned(b)) == 2) r.c[b] = c[b];
    return r;
  }
  Mv even() const {
    Mv r;
    for (int b = 0; b < DIM; ++b) if ((popc(unsigned(b)) & 1) == 0) r.c[b] = c[b];
    return r;
  }
};

template <class T> struct V3 {
  T x[3];
  V3() { x[0] = x[1] = x[2] = T(0.0); }
  V3(T a, T b, T c) { x[0] = a; x[1] = b; x[2] = c; }
  T& operator[](int i) { return x[i]; }
  const T& operator[](int i) const { return x[i]; }
  V3 operator+(const V3& o) const { return V3(x[0] + o.x[0], x[1] + o.x[1], x[2] + o.x[2]); }
  V3 operator-(const V3& o) const { return V3(x[0] - o.x[0], x[1] - o.x[1], x[2] - o.x[2]); }
  V3 operator-() const { return V3(-x[0], -x[1], -x[2]); }
  V3 scale(const T& s) const { return V3(x[0] * s, x[1] * s, x[2] * s); }
  T dot(const V3& o) const { return x[0] * o.x[0] + x[1] * o.x[1] + x[2] * o.x[2]; }
  V3 cross(const V3& o) const {
    return V3(x[1] * o.x[2] - x[2] * o.x[1], x[2] * o.x[0] - x[0] * o.x[2], x[0] * o.x[1] - x[1] * o.x[0]);
  }
};

// Dual readers/writers of physical quantities (mv.rs:527-560, 619-705).
template <class T, class F> V3<T> read_dual(const Mv<T>& m, F blade) {
  V3<T> out;
  for (int i = 0; i < 3; ++i) { MaskSign ms = blade(i); out[i] = ms.sign < 0 ? -m.c[ms.mask] : m.c[ms.mask]; }
  return out;
}
template <class T, class F> void write_dual(Mv<T>& m, const V3<T>& v, F blade) {
  for (int i = 0; i < 3; ++i) { MaskSign ms = blade(i); m.c[ms.mask] = m.c[ms.mask] + (ms.sign < 0 ? -v[i] : v[i]); }
}

}  // namespace oracle
