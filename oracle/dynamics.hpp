// ORACLE — test infrastructure only (CPU restatement the CUDA path is checked against).
// Pinned against the reference's own known-answer tests and test properties, restated with their
// file:line in tests/test_oracle_kat.py, tests/test_oracle_world_kats.py and
// tests/test_seam_oracle.py (the reference keeps no golden vectors and cannot be built here).
//
// f64 restatement of the per-step dynamics path, composed in the reference's order:
//   * RigidBody state: pose motor + BODY-frame momentum (crates/newton/src/body.rs:32-205),
//     inertia apply / apply_inverse (crates/newton/src/inertia.rs:271-345);
//   * gravity: the reference's size-core law `pair_force` (crates/newton/src/gravity.rs:110-140)
//     and the Plummer-softened law of the synthetic configs; the wrench on a body is
//     (F, p x F) (gravity.rs:593-601), here about the world origin;
//   * explicit step: bridge::explicit_step_all (crates/newton/src/integrator/implicit/bridge.rs:19-63)
//     with ExplicitEuler / SymplecticEuler / LieEuler (integrator/explicit/*.rs);
//   * implicit mid-point Newton: Newton::step_all / solve_step / newton_solve /
//     commit_span (crates/newton/src/integrator/implicit/newton.rs:334-861), stage bodies from
//     crates/functions/src/lib.rs:15-247, assembly per crates/newton/src/accelerator/rows/assemble.rs.
//     The linear solve is pluggable: SOLVER_EXACT (block elimination on the island tree,
//     dense LU for cyclic islands) or SOLVER_REFERENCE_NS (the reference's dense-block
//     Newton-Schulz with warm / seed budgets, reseed guard and accepted-X rollback,
//     newton.rs:209-327, cache.rs:543-560, 1154-1172).
// Poses are held in absolute world coordinates. The reference re-anchors each island's
// poses on its centre of mass after every step (mechanism/island.rs:206-243); that is a
// change of representation with no physical effect and is not repeated here.
#pragma once
#include <algorithm>
#include <cstring>
#include <functional>
#include <limits>
#include <omp.h>
#include <vector>
#include "laws.hpp"

namespace oracle {

typedef std::array<double, 36> Block;  // [row][col], row-major

struct OBody {
  double pose[8];
  double mom[6];      // body-frame momentum (force, torque)
  double mass;
  double inertia[9];  // 3x3 angular inertia tensor, row-major
  int diag;           // 1: diagonal tensor (only the diagonal is read)
  int kinematic;
  double size;        // effective size (m/4)^(1/3) unless overridden
};
struct OJoint { int law, a, b; double p[10]; };

enum Integrator { EXPLICIT_EULER = 0, SYMPLECTIC_EULER = 1, LIE_EULER = 2, NEWTON = 3 };
enum GravityLaw { GRAVITY_OFF = 0, GRAVITY_SIZE_CORE = 1, GRAVITY_PLUMMER = 2 };
enum Solver { SOLVER_EXACT = 0, SOLVER_REFERENCE_NS = 1 };
constexpr double kFrameGrid = 1024.0;  // island frames' anchors lie on this grid (NewtonIsland::make_frame)

// body.rs:70-77
inline double effective_size(double mass) { return std::pow(mass / 4.0, 1.0 / 3.0); }

// ── Inertia (inertia.rs:271-345) ─────────────────────────────────────────────
inline Wrench<double> inertia_apply(const OBody& b, const Twist<double>& t) {
  if (b.kinematic) return Wrench<double>::make(t.lin(), t.ang());
  V3<double> v = t.lin(), w = t.ang();
  V3<double> l;
  if (b.diag) l = V3<double>(b.inertia[0] * w[0], b.inertia[4] * w[1], b.inertia[8] * w[2]);
  else {
    const double* a = b.inertia;
    l = V3<double>(a[0] * w[0] + a[1] * w[1] + a[2] * w[2], a[3] * w[0] + a[4] * w[1] + a[5] * w[2],
                   a[6] * w[0] + a[7] * w[1] + a[8] * w[2]);
  }
  return Wrench<double>::make(v.scale(b.mass), l);
}
// inertia.rs:12-45: 3x3 solve through cofactors
inline V3<double> solve3(const double* a, const V3<double>& b) {
  double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
  double c10 = a[2] * a[7] - a[1] * a[8], c11 = a[0] * a[8] - a[2] * a[6], c12 = a[1] * a[6] - a[0] * a[7];
  double c20 = a[1] * a[5] - a[2] * a[4], c21 = a[2] * a[3] - a[0] * a[5], c22 = a[0] * a[4] - a[1] * a[3];
  double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  return V3<double>((c00 * b[0] + c10 * b[1] + c20 * b[2]) / det, (c01 * b[0] + c11 * b[1] + c21 * b[2]) / det,
                    (c02 * b[0] + c12 * b[1] + c22 * b[2]) / det);
}
inline Twist<double> inertia_apply_inverse(const OBody& b, const Wrench<double>& p) {
  if (b.kinematic) return Twist<double>::make(p.lin(), p.ang());
  V3<double> f = p.lin(), t = p.ang();
  V3<double> w;
  if (b.diag) w = V3<double>(t[0] / b.inertia[0], t[1] / b.inertia[4], t[2] / b.inertia[8]);
  else w = solve3(b.inertia, t);
  return Twist<double>::make(f.scale(1.0 / b.mass), w);
}

inline Motor<double> body_pose(const OBody& b) { return Motor<double>::from_components(b.pose); }
inline Wrench<double> body_mom(const OBody& b) { return Wrench<double>::from6(b.mom); }
inline Twist<double> body_velocity(const OBody& b) { return inertia_apply_inverse(b, body_mom(b)); }
// body.rs:141-148 / 180-186
inline Twist<double> world_velocity(const OBody& b) { return body_velocity(b).transport_contra(body_pose(b)); }
inline Wrench<double> world_momentum(const OBody& b) { return body_mom(b).transport_co(body_pose(b)); }
inline V3<double> body_position(const OBody& b) { Point<double> p = anchor_point(body_pose(b), V3<double>()); return p.coords(); }
// body.rs:170-175
inline Wrench<double> gyroscopic(const OBody& b) { return -coad_bracket(body_mom(b), body_velocity(b)); }
inline double kinetic_energy(const OBody& b) { return 0.5 * power(body_mom(b), body_velocity(b)); }

// ── Gravity ──────────────────────────────────────────────────────────────────
// gravity.rs:110-140, literally through the algebra: force on `lo` from `hi`, or false if
// coincident. Used by tests to pin the closed form below.
inline bool pair_force_literal(const V3<double>& p_lo, double g_lo, const V3<double>& p_hi, double g_hi, double size_hi,
                               V3<double>& out) {
  M<double> line = Point<double>::at(p_lo).join(Point<double>::at(p_hi));
  double d = line_weight_norm(line);
  if (eff_zero(d)) return false;
  double g;
  if (d >= size_hi) g = (g_lo / d) * (g_hi / d) / d;
  else g = (g_lo / size_hi) * (g_hi / size_hi) / size_hi;
  out = from_line(line).scale(-g).lin();
  return true;
}

struct GravityParams { int law; double G; double eps; };

// Per-body world force from every other body, summed in slot order (gravity.rs:530-587,
// 438-450). SIZE_CORE: the reference law with the higher-slot body's size as the core.
// PLUMMER: F = G m_i m_j (p_j - p_i) / (r^2 + eps^2)^(3/2).
// Host threads the oracle may use (OpenMP): over gravity rows, over the islands of a world, over
// an island's joints and bodies, and over worlds (orc_worlds_step). Every parallel loop writes
// disjoint outputs and every reduction runs serially in index order afterwards, so results do not
// depend on the thread count.
inline int& oracle_threads() { static int t = 1; return t; }

inline void gravity_forces(const std::vector<OBody>& bodies, const GravityParams& gp, std::vector<V3<double>>& force) {
  size_t n = bodies.size();
  force.assign(n, V3<double>());
  if (gp.law == GRAVITY_OFF) return;
  std::vector<V3<double>> pos(n);
  for (size_t i = 0; i < n; ++i) pos[i] = body_position(bodies[i]);
  const int nt = std::max(1, std::min<int>(oracle_threads(), (int)n));
#pragma omp parallel for schedule(static) num_threads(nt) if (nt > 1 && !omp_in_parallel())
  for (long long ii = 0; ii < (long long)n; ++ii) {
    const size_t i = (size_t)ii;
    if (bodies[i].kinematic) continue;
    double mi = bodies[i].mass;
    V3<double> acc;
    for (size_t j = 0; j < n; ++j) {
      if (j == i || bodies[j].kinematic) continue;
      double mj = bodies[j].mass;
      V3<double> r = pos[j] - pos[i];
      double r2 = r.dot(r);
      if (gp.law == GRAVITY_PLUMMER) {
        double s2 = r2 + gp.eps * gp.eps;
        double inv = 1.0 / (s2 * std::sqrt(s2));
        acc = acc + r.scale(gp.G * mi * mj * inv);
      } else {
        double d = std::sqrt(r2);
        if (eff_zero(d)) continue;
        double size_hi = bodies[std::max(i, j)].size;
        double core = d >= size_hi ? d : size_hi;
        acc = acc + r.scale(gp.G * mi * mj / (core * core * core));
      }
    }
    force[i] = acc;
  }
}

inline double gravity_potential(const std::vector<OBody>& bodies, const GravityParams& gp) {
  if (gp.law == GRAVITY_OFF) return 0.0;
  size_t n = bodies.size();
  std::vector<V3<double>> pos(n);
  for (size_t i = 0; i < n; ++i) pos[i] = body_position(bodies[i]);
  // per-row sums in parallel, then the rows in order
  std::vector<double> row(n, 0.0);
  const int nt = std::max(1, std::min<int>(oracle_threads(), (int)n));
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt) if (nt > 1 && !omp_in_parallel())
  for (long long ii = 0; ii < (long long)n; ++ii) {
    const size_t i = (size_t)ii;
    double e = 0.0;
    for (size_t j = i + 1; j < n; ++j) {
      if (bodies[i].kinematic || bodies[j].kinematic) continue;
      V3<double> r = pos[j] - pos[i];
      double r2 = r.dot(r), mm = gp.G * bodies[i].mass * bodies[j].mass;
      if (gp.law == GRAVITY_PLUMMER) e -= mm / std::sqrt(r2 + gp.eps * gp.eps);
      else {
        double d = std::sqrt(r2), s = bodies[j].size;
        e -= d >= s ? mm / d : mm * (3.0 * s * s - r2) / (2.0 * s * s * s);
      }
    }
    row[i] = e;
  }
  double e = 0.0;
  for (size_t i = 0; i < n; ++i) e += row[i];
  return e;
}

// ── Islands (connected components of the joint graph) ───────────────────────
struct Island {
  std::vector<int> bodies;  // ascending body index
  std::vector<int> joints;  // ascending joint index
  std::vector<int> order;   // position in the solve per island body, -1 for kinematic
  int m = 0;                // dynamic bodies
  // reference Newton-Schulz state (SOLVER_REFERENCE_NS), persistent across steps
  std::vector<Block> X, X_accepted;
  bool seeded = false, accepted_seeded = false;
  int last_spans = 0;
  int last_newton_iterations = 0;
};

inline std::vector<Island> build_islands(int n_bodies, const std::vector<OJoint>& joints, const std::vector<OBody>& bodies) {
  std::vector<int> parent(n_bodies);
  for (int i = 0; i < n_bodies; ++i) parent[i] = i;
  std::function<int(int)> find = [&](int x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
  for (const OJoint& j : joints) { int ra = find(j.a), rb = find(j.b); if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb); }
  std::vector<int> island_of_root(n_bodies, -1);
  std::vector<Island> out;
  for (int i = 0; i < n_bodies; ++i) {
    int r = find(i);
    if (island_of_root[r] < 0) { island_of_root[r] = (int)out.size(); out.emplace_back(); }
    out[island_of_root[r]].bodies.push_back(i);
  }
  for (size_t k = 0; k < joints.size(); ++k) out[island_of_root[find(joints[k].a)]].joints.push_back((int)k);
  for (Island& isl : out) {
    isl.order.assign(isl.bodies.size(), -1);
    int m = 0;
    for (size_t q = 0; q < isl.bodies.size(); ++q) if (!bodies[isl.bodies[q]].kinematic) isl.order[q] = m++;
    isl.m = m;
  }
  return out;
}

// bake_incidence (crates/newton/src/accelerator/mod.rs:289-331; the solver cache's gather terms
// follow the same order, integrator/implicit/cache.rs:885-897): per island body, the joint wrench
// slots flowing into its total, in joint traversal order, end a (slot 0) before end b (slot 1).
// CSR over island bodies: ptr[q] .. ptr[q+1] index `ref`, each entry island joint * 2 + slot.
inline void bake_incidence(const Island& isl, const std::vector<OJoint>& joints, std::vector<int>& ptr,
                           std::vector<int>& ref) {
  const int n = (int)isl.bodies.size();
  auto local = [&](int g) { return int(std::lower_bound(isl.bodies.begin(), isl.bodies.end(), g) - isl.bodies.begin()); };
  std::vector<std::vector<int>> acc(n);
  for (size_t q = 0; q < isl.joints.size(); ++q) {
    const OJoint& j = joints[isl.joints[q]];
    acc[local(j.a)].push_back(2 * (int)q + 0);
    acc[local(j.b)].push_back(2 * (int)q + 1);
  }
  ptr.assign(1, 0);
  ref.clear();
  for (int q = 0; q < n; ++q) {
    ref.insert(ref.end(), acc[q].begin(), acc[q].end());
    ptr.push_back((int)ref.size());
  }
}

// ── Explicit integrators (integrator/explicit/*.rs) ─────────────────────────
inline void integrate_explicit(int scheme, OBody& b, const Wrench<double>& w_body, double dt) {
  if (b.kinematic) return;
  Motor<double> pose = body_pose(b);
  Wrench<double> mom = body_mom(b);
  if (scheme == LIE_EULER) {  // lie_euler.rs:31-55
    mom = mom + w_body.scale(dt);
    mom.to6(b.mom);
    Motor<double> delta = twist_exp(body_velocity(b), dt);
    Motor<double> drot = delta.rotation_part();
    mom = mom.transport_co(drot.inverse());
    mom.to6(b.mom);
    pose = delta.compose(pose);
  } else if (scheme == SYMPLECTIC_EULER) {  // symplectic_euler.rs:26-41
    Wrench<double> gyro = gyroscopic(b);
    mom = mom + (w_body + gyro).scale(dt);
    mom.to6(b.mom);
    Twist<double> v_new = body_velocity(b);
    pose = twist_exp(v_new, dt).compose(pose);
  } else {  // explicit_euler.rs:21-33
    Twist<double> v = body_velocity(b);
    Wrench<double> gyro = gyroscopic(b);
    pose = twist_exp(v, dt).compose(pose);
    mom = mom + (w_body + gyro).scale(dt);
    mom.to6(b.mom);
  }
  pose.to_components(b.pose);
}

// Per-body gather (accelerator/mod.rs:289-331): total = external + incident connection
// wrenches, joints in order, end a before end b.
inline void gather_totals(const std::vector<OJoint>& joints, const std::vector<int>& jidx, const std::vector<double>& conn12,
                          std::vector<Wrench<double>>& total) {
  for (size_t q = 0; q < jidx.size(); ++q) {
    const OJoint& j = joints[jidx[q]];
    total[j.a] = total[j.a] + Wrench<double>::from6(&conn12[q * 12]);
    total[j.b] = total[j.b] + Wrench<double>::from6(&conn12[q * 12 + 6]);
  }
}

// ── 6x6 block helpers ─────────────────────────────────────────────────────────
inline Block zero_block() { Block b; b.fill(0.0); return b; }
inline void block_mul_acc(Block& out, const Block& a, const Block& b) {
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) {
      double s = 0.0;
      for (int k = 0; k < 6; ++k) s += a[r * 6 + k] * b[k * 6 + c];
      out[r * 6 + c] += s;
    }
}
inline double fro2(const Block& b) { double s = 0.0; for (double v : b) s += v * v; return s; }
// Gauss-Jordan inverse with partial pivoting; false if singular.
inline bool block_inverse(const Block& a, Block& inv) {
  double m[6][12];
  for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) { m[r][c] = a[r * 6 + c]; m[r][6 + c] = (r == c) ? 1.0 : 0.0; }
  for (int k = 0; k < 6; ++k) {
    int piv = k; double best = std::fabs(m[k][k]);
    for (int r = k + 1; r < 6; ++r) if (std::fabs(m[r][k]) > best) { best = std::fabs(m[r][k]); piv = r; }
    if (best == 0.0 || !std::isfinite(best)) return false;
    if (piv != k) for (int c = 0; c < 12; ++c) std::swap(m[k][c], m[piv][c]);
    double ip = 1.0 / m[k][k];
    for (int c = 0; c < 12; ++c) m[k][c] *= ip;
    for (int r = 0; r < 6; ++r) if (r != k) { double f = m[r][k]; if (f != 0.0) for (int c = 0; c < 12; ++c) m[r][c] -= f * m[k][c]; }
  }
  for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) inv[r * 6 + c] = m[r][6 + c];
  return true;
}


// Block-sparse matrix over the island's dynamic bodies: per row, the blocks of the columns in its
// sparsity pattern (the row itself and its joint neighbours, cache.rs:712-724), columns ascending.
// Absent blocks read as zero, so the dense loops of the solvers below read it unchanged while a
// tree island of m bodies stores O(m) blocks instead of m^2.
struct SparseBlocks {
  int m = 0;
  std::vector<std::vector<int>> cols;
  std::vector<std::vector<Block>> vals;
  void init(int m_, const std::vector<std::vector<int>>& pattern) {
    m = m_;
    cols.assign(m, {});
    vals.assign(m, {});
    for (int i = 0; i < m; ++i) {
      cols[i] = pattern[i];
      std::sort(cols[i].begin(), cols[i].end());
      vals[i].assign(cols[i].size(), zero_block());
    }
  }
  const Block* find(int i, int j) const {
    const std::vector<int>& c = cols[i];
    auto it = std::lower_bound(c.begin(), c.end(), j);
    return (it != c.end() && *it == j) ? &vals[i][it - c.begin()] : nullptr;
  }
  Block& at(int i, int j) { return const_cast<Block&>(*find(i, j)); }  // (i, j) in the pattern
  const Block& get(int i, int j) const {
    static const Block zero = zero_block();
    const Block* b = find(i, j);
    return b ? *b : zero;
  }
};

// functions/src/lib.rs:170-247 — world mass block, residual rhs = -R and self-scale.
inline void body_post(const OBody& b, const Motor<double>& pose_mid, const Twist<double>& solve_vel, const Wrench<double>& snap_mom,
                      const Wrench<double>& total, double half, double floor2, Block& block, double rhs[6], double scale[6]) {
  Motor<double> inv = pose_mid.inverse();
  for (int col = 0; col < 6; ++col) {
    double e[6] = {0, 0, 0, 0, 0, 0}; e[col] = 1.0;
    Twist<double> ej_body = Twist<double>::from6(e).transport_contra(inv);
    V3<double> v = ej_body.lin(), w = ej_body.ang();
    V3<double> l;
    if (b.diag) l = V3<double>(b.inertia[0] * w[0], b.inertia[4] * w[1], b.inertia[8] * w[2]);
    else {
      const double* a = b.inertia;
      l = V3<double>(a[0] * w[0] + a[1] * w[1] + a[2] * w[2], a[3] * w[0] + a[4] * w[1] + a[5] * w[2],
                     a[6] * w[0] + a[7] * w[1] + a[8] * w[2]);
    }
    Wrench<double> column = Wrench<double>::make(v.scale(b.mass), l).transport_co(pose_mid);
    double vals[6]; column.to6(vals);
    for (int r = 0; r < 6; ++r) block[r * 6 + col] = vals[r];
  }
  double v[6]; solve_vel.to6(v);
  double p[6];
  for (int r = 0; r < 6; ++r) { double acc = 0.0; for (int c = 0; c < 6; ++c) acc += block[r * 6 + c] * v[c]; p[r] = acc; }
  double nn[6], hh[6];
  snap_mom.to6(nn);
  total.scale(half).to6(hh);
  for (int r = 0; r < 6; ++r) rhs[r] = -(p[r] - nn[r] - hh[r]);
  auto sq = [](const double* x, int o) { return x[o] * x[o] + x[o + 1] * x[o + 1] + x[o + 2] * x[o + 2]; };
  double lin = std::max(std::max(std::max(sq(p, 0), sq(nn, 0)), sq(hh, 0)), floor2);
  double ang = std::max(std::max(std::max(sq(p, 3), sq(nn, 3)), sq(hh, 3)), floor2);
  scale[0] = scale[1] = scale[2] = lin;
  scale[3] = scale[4] = scale[5] = ang;
}

struct WorldParams {
  int integrator = LIE_EULER;
  GravityParams gravity{GRAVITY_OFF, 1.0, 0.0};
  double dt = 1e-2, warp = 1.0;
  double tol = 1e-4;      // relative per-block Newton tolerance (newton.rs:799-805 uses 1e-4)
  int ns_warm = 2, ns_seed = 24;
  int solver = SOLVER_EXACT;
  bool exact_pose_factor = false;  // -half^2/2 on the pose columns instead of the reference's -half^2
  double field[3] = {0.0, 0.0, 0.0};  // UniformField world acceleration (field.rs:17-47)
};

// ── One island's implicit mid-point Newton step ─────────────────────────────
struct NewtonIsland {
  std::vector<OBody>& bodies;
  const std::vector<OJoint>& joints;
  Island& isl;
  const WorldParams& wp;
  const std::vector<Wrench<double>>& external;  // per global body (world)
  // scratch
  std::vector<Motor<double>> mid;               // per island body
  std::vector<Block> mass;                      // per dynamic body (this evaluation)
  std::vector<double> rhs, scale;               // 6 per dynamic body
  std::vector<double> jac;                      // 300 per island joint
  std::vector<Block> lane0_mass;                // the mass blocks lane 0 last wrote
  SparseBlocks A;                               // last assembled system, block-sparse
  std::vector<std::vector<int>> nbrs;           // sparsity (cache.rs:712-724)
  double a_norm2 = 0.0;
  bool have_A = false;
  int newton_iterations = 0;

  // The step's frame: the island's poses are taken relative to an anchor near its centre of mass at
  // the step's start, delta = sum m_i r_i / M (kinematic bodies weigh nothing; the first body's
  // position where the island has no dynamic mass) rounded to a multiple of kFrameGrid in each
  // component, and written back in world coordinates. The reference re-binds each island's origin
  // to its centre of mass after every step (Island::recompute_centroid, mechanism/island.rs:206-243);
  // the rounding keeps islands within kFrameGrid / 2 of the world origin in world coordinates, where
  // the Newton residual's per-body angular scale (functions/src/lib.rs:170-247) has the lever arms
  // the tolerances here are set for: at the centre of mass itself a small island's angular scale
  // falls to the residual's 1e-9 floor and a 1e-10 tolerance is out of reach.
  std::vector<Motor<double>> lpose;   // per island body, in the island's frame
  std::vector<Wrench<double>> lext;   // external wrenches about the anchor
  Motor<double> to_world;

  NewtonIsland(std::vector<OBody>& b, const std::vector<OJoint>& j, Island& i, const WorldParams& w, const std::vector<Wrench<double>>& e)
      : bodies(b), joints(j), isl(i), wp(w), external(e) {}

  void make_frame() {
    double wx[3] = {0.0, 0.0, 0.0}, total = 0.0;
    for (int q = 0; q < nb(); ++q) {
      const OBody& b = bodies[isl.bodies[q]];
      const double m = b.kinematic ? 0.0 : b.mass;
      const V3<double> r = body_position(b);
      for (int k = 0; k < 3; ++k) wx[k] += r[k] * m;
      total += m;
    }
    V3<double> a = body_position(bodies[isl.bodies[0]]);
    if (total > 0.0) {
      const double inv = 1.0 / total;
      a = V3<double>(wx[0] * inv, wx[1] * inv, wx[2] * inv);
    }
    for (int k = 0; k < 3; ++k) a[k] = kFrameGrid * std::nearbyint(a[k] / kFrameGrid);
    const double neg[6] = {-a[0], -a[1], -a[2], 0.0, 0.0, 0.0}, pos[6] = {a[0], a[1], a[2], 0.0, 0.0, 0.0};
    const Motor<double> to_local = twist_exp(Twist<double>::from6(neg), 1.0);
    to_world = twist_exp(Twist<double>::from6(pos), 1.0);
    lpose.resize(nb());
    lext.resize(nb());
    for (int q = 0; q < nb(); ++q) {
      lpose[q] = body_pose(bodies[isl.bodies[q]]).compose(to_local);
      const Wrench<double>& e = external[isl.bodies[q]];
      double w6[6];
      e.to6(w6);
      const V3<double> f(w6[0], w6[1], w6[2]);
      const V3<double> m = V3<double>(w6[3], w6[4], w6[5]) - a.cross(f);
      lext[q] = Wrench<double>::make(f, m);
    }
  }

  int nb() const { return (int)isl.bodies.size(); }
  int local_of(int global) const { return int(std::lower_bound(isl.bodies.begin(), isl.bodies.end(), global) - isl.bodies.begin()); }

  // PRE + joints (+ Jacobian) + gather + POST at iterate vmid; returns wnorm.
  double evaluate(const std::vector<Twist<double>>& vmid, const std::vector<Wrench<double>>& snap, double half, bool with_jac,
                  std::vector<Block>& mass_out, std::vector<double>& rhs_out, std::vector<double>& scale_out) {
    int n = nb();
    mid.resize(n);
    for (int q = 0; q < n; ++q) mid[q] = lpose[q].compose(twist_exp(vmid[q], half));  // functions::pre
    size_t nj = isl.joints.size();
    std::vector<double> conn(nj * 12);
    if (with_jac) jac.resize(nj * 300);
    const int nt = oracle_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt) if (nt > 1 && nj > 64 && !omp_in_parallel())
    for (long long qq = 0; qq < (long long)nj; ++qq) {
      const size_t q = (size_t)qq;
      const OJoint& j = joints[isl.joints[q]];
      int la = local_of(j.a), lb = local_of(j.b);
      double pa[8], pb[8], va[6], vb[6];
      mid[la].to_components(pa); mid[lb].to_components(pb);
      vmid[la].to6(va); vmid[lb].to6(vb);
      if (with_jac) {
        jacobian_eval(j.law, j.p, pa, pb, va, vb, wp.dt, wp.warp, &jac[q * 300]);
        for (int c = 0; c < 12; ++c) conn[q * 12 + c] = jac[q * 300 + c * 25];
      } else {
        plain_eval(j.law, j.p, pa, pb, va, vb, wp.dt, wp.warp, &conn[q * 12]);
      }
    }
    std::vector<Wrench<double>> total(n);
    for (int q = 0; q < n; ++q) total[q] = lext[q];
    for (size_t q = 0; q < nj; ++q) {
      const OJoint& j = joints[isl.joints[q]];
      int la = local_of(j.a), lb = local_of(j.b);
      total[la] = total[la] + Wrench<double>::from6(&conn[q * 12]);
      total[lb] = total[lb] + Wrench<double>::from6(&conn[q * 12 + 6]);
    }
    int m = isl.m;
    mass_out.resize(m); rhs_out.resize(6 * m); scale_out.resize(6 * m);
    double floor2 = 1e-9 * 1e-9;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt) if (nt > 1 && n > 64 && !omp_in_parallel())
    for (int q = 0; q < n; ++q) {
      int i = isl.order[q];
      if (i < 0) continue;
      body_post(bodies[isl.bodies[q]], mid[q], vmid[q], snap[q], total[q], half, floor2, mass_out[i], &rhs_out[6 * i], &scale_out[6 * i]);
    }
    double worst = 0.0;
    for (int q = 0; q < n; ++q) {
      int i = isl.order[q];
      if (i < 0) continue;
      const double* r = &rhs_out[6 * i];
      double lin2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      double ang2 = r[3] * r[3] + r[4] * r[4] + r[5] * r[5];
      // newton.rs:139-151: max2 with NaN falling through `a > b`
      double a1 = lin2 / scale_out[6 * i], a2 = ang2 / scale_out[6 * i + 3];
      worst = (worst > a1) ? worst : a1;
      worst = (worst > a2) ? worst : a2;
    }
    return worst;
  }

  void build_sparsity() {
    int m = isl.m;
    nbrs.assign(m, {});
    for (int i = 0; i < m; ++i) nbrs[i].push_back(i);
    for (int jq : isl.joints) {
      const OJoint& j = joints[jq];
      int ia = isl.order[local_of(j.a)], ib = isl.order[local_of(j.b)];
      if (ia >= 0 && ib >= 0) {
        if (std::find(nbrs[ia].begin(), nbrs[ia].end(), ib) == nbrs[ia].end()) nbrs[ia].push_back(ib);
        if (std::find(nbrs[ib].begin(), nbrs[ib].end(), ia) == nbrs[ib].end()) nbrs[ib].push_back(ia);
      }
    }
  }

  // rows/assemble.rs + functions::assemble_term: A_ij = [i==j] mass_i + sum over joint ends
  // (pf * pose columns + vf * velocity columns), pf = -half^2, vf = -half.
  void assemble(double half) {
    int m = isl.m;
    A.init(m, nbrs);
    for (int i = 0; i < m; ++i) A.at(i, i) = lane0_mass[i];
    double pf = -(half * half) * (wp.exact_pose_factor ? 0.5 : 1.0), vf = -half;
    for (size_t q = 0; q < isl.joints.size(); ++q) {
      const OJoint& j = joints[isl.joints[q]];
      int ends[2] = {isl.order[local_of(j.a)], isl.order[local_of(j.b)]};
      for (int re = 0; re < 2; ++re) {
        if (ends[re] < 0) continue;
        for (int ce = 0; ce < 2; ++ce) {
          if (ends[ce] < 0) continue;
          Block& out = A.at(ends[re], ends[ce]);
          for (int col = 0; col < 6; ++col)
            for (int r = 0; r < 6; ++r) {
              int comp = re * 6 + r;
              double p = jac[q * 300 + comp * 25 + 1 + ce * 6 + col];
              double v = jac[q * 300 + comp * 25 + 1 + 12 + ce * 6 + col];
              out[r * 6 + col] = out[r * 6 + col] + pf * p + vf * v;
            }
        }
      }
    }
    a_norm2 = 0.0;
    for (int i = 0; i < m; ++i)  // row-major over (i, j): absent (zero) blocks add nothing
      for (const Block& b : A.vals[i]) a_norm2 += fro2(b);
    have_A = true;
  }

  // ── exact solve: tree elimination, or dense LU for a cyclic island ──
  bool solve_exact(const std::vector<double>& rhs_in, std::vector<double>& dv) {
    int m = isl.m;
    dv.assign(6 * m, 0.0);
    if (m == 0) return true;
    int edges = 0;
    for (int i = 0; i < m; ++i) edges += (int)nbrs[i].size() - 1;
    edges /= 2;
    // connected dynamic graph with m-1 edges is a tree
    std::vector<int> parent(m, -2), bfs;
    bfs.reserve(m);
    parent[0] = -1; bfs.push_back(0);
    for (size_t h = 0; h < bfs.size(); ++h)
      for (size_t k = 1; k < nbrs[bfs[h]].size(); ++k) { int c = nbrs[bfs[h]][k]; if (parent[c] == -2) { parent[c] = bfs[h]; bfs.push_back(c); } }
    bool tree = (edges == m - 1) && ((int)bfs.size() == m);
    if (tree) {
      std::vector<Block> D(m), Dinv(m);
      std::vector<double> b(rhs_in);
      for (int i = 0; i < m; ++i) D[i] = A.get(i, i);
      for (int h = m - 1; h >= 1; --h) {  // leaves first
        int i = bfs[h], p = parent[i];
        if (!block_inverse(D[i], Dinv[i])) return false;
        const Block& Api = A.get(p, i);
        const Block& Aip = A.get(i, p);
        Block S = zero_block();  // Api * Dinv_i
        block_mul_acc(S, Api, Dinv[i]);
        Block T = zero_block();
        block_mul_acc(T, S, Aip);
        for (int k = 0; k < 36; ++k) D[p][k] -= T[k];
        for (int r = 0; r < 6; ++r) { double s = 0.0; for (int c = 0; c < 6; ++c) s += S[r * 6 + c] * b[6 * i + c]; b[6 * p + r] -= s; }
      }
      if (!block_inverse(D[bfs[0]], Dinv[bfs[0]])) return false;
      for (int h = 0; h < m; ++h) {  // root first
        int i = bfs[h], p = parent[i];
        double y[6];
        for (int r = 0; r < 6; ++r) y[r] = b[6 * i + r];
        if (p >= 0) {
          const Block& Aip = A.get(i, p);
          for (int r = 0; r < 6; ++r) { double s = 0.0; for (int c = 0; c < 6; ++c) s += Aip[r * 6 + c] * dv[6 * p + c]; y[r] -= s; }
        }
        for (int r = 0; r < 6; ++r) { double s = 0.0; for (int c = 0; c < 6; ++c) s += Dinv[i][r * 6 + c] * y[c]; dv[6 * i + r] = s; }
      }
      return true;
    }
    int n = 6 * m;
    std::vector<double> a((size_t)n * n), x(rhs_in);
    for (int bi = 0; bi < m; ++bi) for (int bj = 0; bj < m; ++bj)
      for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) a[(size_t)(6 * bi + r) * n + 6 * bj + c] = A.get(bi, bj)[r * 6 + c];
    for (int k = 0; k < n; ++k) {
      int piv = k; double best = std::fabs(a[(size_t)k * n + k]);
      for (int r = k + 1; r < n; ++r) if (std::fabs(a[(size_t)r * n + k]) > best) { best = std::fabs(a[(size_t)r * n + k]); piv = r; }
      if (best == 0.0 || !std::isfinite(best)) return false;
      if (piv != k) { for (int c = 0; c < n; ++c) std::swap(a[(size_t)k * n + c], a[(size_t)piv * n + c]); std::swap(x[k], x[piv]); }
      for (int r = k + 1; r < n; ++r) {
        double f = a[(size_t)r * n + k] / a[(size_t)k * n + k];
        if (f == 0.0) continue;
        for (int c = k; c < n; ++c) a[(size_t)r * n + c] -= f * a[(size_t)k * n + c];
        x[r] -= f * x[k];
      }
    }
    for (int k = n - 1; k >= 0; --k) { double s = x[k]; for (int c = k + 1; c < n; ++c) s -= a[(size_t)k * n + c] * x[c]; x[k] = s / a[(size_t)k * n + k]; }
    for (int k = 0; k < n; ++k) dv[k] = x[k];
    return true;
  }

  // ── the reference's dense-block Newton-Schulz (newton.rs:209-327) ──
  void seed_transpose() {
    int m = isl.m;
    double one = 0.0, inf = 0.0;
    for (int i = 0; i < m; ++i) {
      double row = 0.0, col = 0.0;
      for (int j = 0; j < m; ++j) {
        const Block& rb = A.get(i, j);
        const Block& cb = A.get(j, i);
        for (int k = 0; k < 36; ++k) { row += std::fabs(rb[k]); col += std::fabs(cb[k]); }
      }
      inf = (inf > row) ? inf : row;
      one = (one > col) ? one : col;
    }
    double s = 1.0 / (one * inf);
    isl.X.assign((size_t)m * m, zero_block());
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        const Block& src = A.get(j, i);
        Block& dst = isl.X[(size_t)i * m + j];
        for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) dst[r * 6 + c] = src[c * 6 + r] * s;
      }
    isl.seeded = true;
  }
  double refine_inverse() {
    int m = isl.m;
    std::vector<Block> R((size_t)m * m, zero_block());
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        Block acc = zero_block();
        for (int k : nbrs[i]) block_mul_acc(acc, A.get(i, k), isl.X[(size_t)k * m + j]);
        R[(size_t)i * m + j] = acc;
      }
    double contraction = 0.0;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        const Block& b = R[(size_t)i * m + j];
        double diag = (i == j) ? 1.0 : 0.0;
        for (int r = 0; r < 6; ++r) for (int c = 0; c < 6; ++c) { double e = (r == c) ? diag - b[r * 6 + c] : -b[r * 6 + c]; contraction += e * e; }
      }
    std::vector<Block> Xn((size_t)m * m, zero_block());
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        Block acc = zero_block();
        for (int k = 0; k < m; ++k) {
          Block right;
          for (int q = 0; q < 36; ++q) right[q] = -R[(size_t)k * m + j][q];
          if (k == j) for (int r = 0; r < 6; ++r) right[r * 6 + r] += 2.0;
          block_mul_acc(acc, isl.X[(size_t)i * m + k], right);
        }
        Xn[(size_t)i * m + j] = acc;
      }
    isl.X.swap(Xn);
    return contraction;
  }
  void run_budget(int budget, int seed_budget) {
    double margin = 4.0;
    bool have_prev = false, reseeded = false;
    double prev = 0.0;
    int remaining = budget;
    while (remaining > 0) {
      --remaining;
      double before = refine_inverse();
      if (have_prev && !(before < margin * prev) && !reseeded) {
        seed_transpose();
        reseeded = true; have_prev = false; remaining = seed_budget;
        continue;
      }
      prev = before; have_prev = true;
    }
  }
  void solve_ns(const std::vector<double>& rhs_in, std::vector<double>& dv) {
    int m = isl.m;
    if ((int)isl.X.size() != m * m) { isl.X.assign((size_t)m * m, zero_block()); isl.X_accepted = isl.X; isl.seeded = isl.accepted_seeded = false; }
    int budget;
    if (isl.seeded) budget = wp.ns_warm;
    else { seed_transpose(); budget = wp.ns_seed; }
    run_budget(budget, wp.ns_seed);
    dv.assign(6 * m, 0.0);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        const Block& x = isl.X[(size_t)i * m + j];
        for (int r = 0; r < 6; ++r) { double s = 0.0; for (int c = 0; c < 6; ++c) s += x[r * 6 + c] * rhs_in[6 * j + c]; dv[6 * i + r] += s; }
      }
  }

  struct SolveResult { bool converged; double best; std::vector<Twist<double>> vmid; bool assembled; };

  SolveResult newton_solve(const std::vector<Wrench<double>>& snap, double half) {
    const double huge = 1e9;
    const double tol2 = wp.tol * wp.tol;
    int n = nb(), m = isl.m;
    std::vector<Twist<double>> vmid(n);
    for (int q = 0; q < n; ++q) vmid[q] = body_velocity(bodies[isl.bodies[q]]).transport_contra(lpose[q]);
    auto read_vals = [&]() { return vmid; };
    double best = huge;
    std::vector<Twist<double>> best_vals = read_vals();
    bool converged = false, assembled = false;
    std::vector<Block> mass_tmp;
    std::vector<double> rhs_tmp, scale_tmp;
    for (int iter = 0; iter < 32; ++iter) {
      ++newton_iterations;
      double rnorm = evaluate(vmid, snap, half, true, mass, rhs, scale);
      lane0_mass = mass;
      if (rnorm < best) { best = rnorm; best_vals = read_vals(); }
      if (rnorm <= tol2) { converged = true; break; }
      if (!(rnorm < huge)) break;
      assemble(half);
      assembled = true;
      std::vector<double> dv;
      if (wp.solver == SOLVER_REFERENCE_NS) solve_ns(rhs, dv);
      else if (!solve_exact(rhs, dv)) { dv.assign(6 * m, std::numeric_limits<double>::quiet_NaN()); }
      bool no_correction = true;
      for (double x : dv) if (x != 0.0) { no_correction = false; break; }
      if (no_correction) break;
      std::vector<Twist<double>> base = vmid;
      double alpha = 1.0;
      int accepted = -1;
      for (int lane = 0; lane < 8; ++lane) {
        std::vector<Twist<double>> trial = base;
        for (int q = 0; q < n; ++q) {
          int i = isl.order[q];
          if (i < 0) continue;
          trial[q] = base[q] + Twist<double>::from6(&dv[6 * i]).scale(alpha);
        }
        double tnorm = evaluate(trial, snap, half, false, mass_tmp, rhs_tmp, scale_tmp);
        if (lane == 0) lane0_mass = mass_tmp;
        if (tnorm < rnorm) { accepted = lane; vmid = trial; lane0_mass = mass_tmp; break; }
        alpha = alpha / 2.0;
      }
      if (accepted < 0) { vmid = base; break; }
    }
    return {converged, best, best_vals, assembled};
  }

  static bool log2_floor(double v, int& e) {
    if (!(v > 0.0)) return false;
    double x = v; e = 0;
    while (x >= 2.0) { x /= 2.0; ++e; if (e > 250) return false; }
    while (x < 1.0 && e > -250) { x *= 2.0; --e; }
    return true;
  }
  bool signal_log2(bool assembled, int& r) {
    if (!assembled) return false;
    double massn = 0.0;
    for (const Block& b : lane0_mass) massn += fro2(b);
    double stiff = eff_zero(massn) ? 0.0 : a_norm2 / massn;
    return log2_floor(stiff, r);
  }
  static int div_euclid(int a, int b) { int q = a / b; if (a % b < 0) q -= 1; return q; }

  void commit_span(const std::vector<Wrench<double>>& snap, const std::vector<Twist<double>>& vmid, double span, double half, bool converged) {
    for (int q = 0; q < nb(); ++q) {
      if (isl.order[q] < 0) continue;
      OBody& b = bodies[isl.bodies[q]];
      Motor<double> m_start = lpose[q];
      Motor<double> pose_mid = m_start.compose(twist_exp(vmid[q], half));
      Twist<double> v_body = vmid[q].transport_contra(pose_mid.inverse());
      Wrench<double> p_s_mid = inertia_apply(b, v_body).transport_co(pose_mid);
      Wrench<double> p_new = converged ? p_s_mid.scale(2.0) - snap[q] : p_s_mid;
      Motor<double> m_new = m_start.compose(twist_exp(vmid[q], span));
      lpose[q] = m_new;
      m_new.compose(to_world).to_components(b.pose);
      p_new.transport_co(m_new.inverse()).to6(b.mom);
    }
  }

  void checkpoint() {
    if (wp.solver != SOLVER_REFERENCE_NS) return;
    isl.X_accepted = isl.X;
    double n = 0.0;
    for (const Block& b : isl.X) n += fro2(b);
    if (n < 1e18) isl.accepted_seeded = isl.seeded;
    else { isl.seeded = false; isl.accepted_seeded = false; }
  }
  void rollback() {
    if (wp.solver != SOLVER_REFERENCE_NS) return;
    isl.X = isl.X_accepted;
    isl.seeded = isl.accepted_seeded;
  }

  // newton.rs:543-683
  void step(double dt) {
    const int MAX_DEPTH = 8, THRESHOLD_LOG2 = 8, PER_HALVING_LOG2 = 4;
    const double huge = 1e9;
    build_sparsity();
    make_frame();
    if (wp.solver == SOLVER_REFERENCE_NS && (int)isl.X.size() != isl.m * isl.m) {
      isl.X.assign((size_t)isl.m * isl.m, zero_block()); isl.X_accepted = isl.X; isl.seeded = isl.accepted_seeded = false;
    }
    uint64_t remaining = 1ull << MAX_DEPTH;
    int depth = 0, spans = 0;
    newton_iterations = 0;
    while (remaining > 0) {
      uint64_t units = 1ull << (MAX_DEPTH - depth);
      while (units > remaining) { ++depth; units >>= 1; }
      double span = dt;
      for (int k = 0; k < depth; ++k) span = span / 2.0;
      double half = span / 2.0;
      ++spans;
      std::vector<Wrench<double>> snap(nb());
      for (int q = 0; q < nb(); ++q) snap[q] = body_mom(bodies[isl.bodies[q]]).transport_co(lpose[q]);
      SolveResult res = newton_solve(snap, half);
      bool finite = res.best < huge;
      bool last = depth == MAX_DEPTH;
      if (!res.converged && !last) {
        rollback();
        int r, down;
        if (signal_log2(res.assembled, r)) down = div_euclid(r - THRESHOLD_LOG2, PER_HALVING_LOG2) + 1; else down = 1;
        depth += std::min(std::max(down, 1), MAX_DEPTH - depth);
        continue;
      }
      if (res.converged || finite) {
        commit_span(snap, res.vmid, span, half, res.converged);
        checkpoint();
      } else {
        rollback();
      }
      remaining -= units;
      auto aligned = [&](int d) {
        if (d <= 0) return false;
        uint64_t bigger = 1ull << (MAX_DEPTH - (d - 1));
        return bigger <= remaining && remaining % bigger == 0;
      };
      int r;
      if (remaining > 0 && res.converged && aligned(depth) && signal_log2(res.assembled, r)) {
        int up = div_euclid(THRESHOLD_LOG2 - r, PER_HALVING_LOG2);
        while (up > 0 && aligned(depth)) { --depth; --up; }
      }
    }
    isl.last_spans = spans;
    isl.last_newton_iterations = newton_iterations;
  }
};

// ── The world step (mechanism.rs:526-602) ───────────────────────────────────
struct OWorld {
  std::vector<OBody> bodies;
  std::vector<OJoint> joints;
  WorldParams wp;
  std::vector<Island> islands;
  bool built = false;

  void build() { islands = build_islands((int)bodies.size(), joints, bodies); built = true; }

  void step() {
    if (!built) build();
    size_t n = bodies.size();
    // external wrenches: gravity from the state at the start of the step (all islands read
    // the same charge snapshot), as (F, p x F) in the world frame.
    std::vector<V3<double>> f;
    gravity_forces(bodies, wp.gravity, f);
    std::vector<Wrench<double>> external(n);
    for (size_t i = 0; i < n; ++i) {
      if (wp.gravity.law == GRAVITY_OFF) continue;
      V3<double> p = body_position(bodies[i]);
      external[i] = Wrench<double>::make(f[i], p.cross(f[i]));
    }
    // UniformField (field.rs:29-47): F = m a on every body (kinematic bodies have mass 0), added
    // after gravity as a force through the body's centre: (F, p x F) about the world origin.
    if (wp.field[0] != 0.0 || wp.field[1] != 0.0 || wp.field[2] != 0.0) {
      for (size_t i = 0; i < n; ++i) {
        if (bodies[i].kinematic) continue;
        const double m = bodies[i].mass;
        V3<double> F{m * wp.field[0], m * wp.field[1], m * wp.field[2]};
        V3<double> p = body_position(bodies[i]);
        external[i] = external[i] + Wrench<double>::make(F, p.cross(F));
      }
    }
    if (wp.integrator == NEWTON) {
      const int nt = oracle_threads(), ni_count = (int)islands.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) if (nt > 1 && ni_count > 1 && !omp_in_parallel())
      for (int k = 0; k < ni_count; ++k) {
        NewtonIsland ni(bodies, joints, islands[k], wp, external);
        ni.step(wp.dt);
      }
      return;
    }
    // explicit family (bridge.rs:19-63): plain joints at the current pose / world velocity
    std::vector<Wrench<double>> total(external);
    std::vector<double> conn(joints.size() * 12);
    std::vector<int> jidx(joints.size());
    for (size_t q = 0; q < joints.size(); ++q) {
      jidx[q] = (int)q;
      const OJoint& j = joints[q];
      double pa[8], pb[8], va[6], vb[6];
      std::memcpy(pa, bodies[j.a].pose, sizeof pa);
      std::memcpy(pb, bodies[j.b].pose, sizeof pb);
      world_velocity(bodies[j.a]).to6(va);
      world_velocity(bodies[j.b]).to6(vb);
      plain_eval(j.law, j.p, pa, pb, va, vb, wp.dt, wp.warp, &conn[q * 12]);
    }
    gather_totals(joints, jidx, conn, total);
    for (size_t i = 0; i < n; ++i) {
      OBody& b = bodies[i];
      Wrench<double> w_body = total[i].transport_co(body_pose(b).inverse());
      integrate_explicit(wp.integrator, b, w_body, wp.dt);
    }
  }

  double energy() const {
    double e = 0.0;
    for (const OBody& b : bodies) if (!b.kinematic) e += kinetic_energy(b);
    e += gravity_potential(bodies, wp.gravity);
    for (const OJoint& j : joints) e += law_potential(j.law, j.p, body_pose(bodies[j.a]), body_pose(bodies[j.b]));
    return e;
  }
};

}  // namespace oracle
