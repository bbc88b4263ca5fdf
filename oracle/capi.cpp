// ORACLE — test infrastructure only. C entry points over the f64 restatement, loaded by the
// test suite (ctypes) to check the CUDA path; the shipped library never links this.
// Records use the public layouts of include/exg.h so one numpy array feeds both sides.
#include <algorithm>
#include <cstring>
#include <new>
#include "../include/exg.h"
#include "dynamics.hpp"

using namespace oracle;

namespace {
OBody to_obody(const exg_body_t& b) {
  OBody o;
  std::memcpy(o.pose, b.pose, sizeof o.pose);
  std::memcpy(o.mom, b.momentum, sizeof o.mom);
  o.mass = b.mass;
  std::memcpy(o.inertia, b.inertia, sizeof o.inertia);
  o.diag = b.diagonal;
  o.kinematic = b.kinematic;
  o.size = b.size;
  return o;
}
void from_obody(const OBody& o, exg_body_t& b) {
  std::memcpy(b.pose, o.pose, sizeof o.pose);
  std::memcpy(b.momentum, o.mom, sizeof o.mom);
  b.mass = o.mass;
  std::memcpy(b.inertia, o.inertia, sizeof o.inertia);
  b.diagonal = o.diag;
  b.kinematic = o.kinematic;
  b.size = o.size;
}
}  // namespace

extern "C" {

void orc_set_threads(int n) { oracle_threads() = n > 0 ? n : 1; }
int orc_body_size(void) { return (int)sizeof(exg_body_t); }
int orc_joint_size(void) { return (int)sizeof(exg_joint_t); }

void* orc_world_create(const exg_body_t* bodies, int n_bodies, const exg_joint_t* joints, int n_joints,
                       const exg_step_params_t* p, int solver, int ns_warm, int ns_seed) {
  OWorld* w = new (std::nothrow) OWorld();
  if (!w) return nullptr;
  for (int i = 0; i < n_bodies; ++i) w->bodies.push_back(to_obody(bodies[i]));
  for (int k = 0; k < n_joints; ++k) {
    OJoint j;
    j.law = joints[k].law; j.a = joints[k].a; j.b = joints[k].b;
    std::memcpy(j.p, joints[k].params, sizeof j.p);
    w->joints.push_back(j);
  }
  w->wp.integrator = p->integrator;
  w->wp.gravity = GravityParams{p->gravity_law, p->G, p->softening};
  w->wp.dt = p->dt;
  w->wp.warp = p->warp;
  w->wp.tol = p->tol;
  w->wp.solver = solver;
  w->wp.ns_warm = ns_warm;
  w->wp.ns_seed = ns_seed;
  w->wp.exact_pose_factor = (p->newton_flags & EXG_NEWTON_EXACT_POSE_FACTOR) != 0;
  for (int k = 0; k < 3; ++k) w->wp.field[k] = p->field_accel[k];
  w->build();
  return w;
}
void orc_world_destroy(void* h) { delete static_cast<OWorld*>(h); }
// Step n_worlds independent worlds `steps` times each on the oracle's threads: worlds of at least
// kBigWorld bodies one after another, each using every thread inside (gravity rows, islands,
// joints), then the smaller worlds spread over the threads one world per thread (largest first).
void orc_worlds_step(void** handles, int n_worlds, int steps) {
  constexpr size_t kBigWorld = 512;
  const int nt = oracle_threads();
  std::vector<OWorld*> big, small;
  for (int k = 0; k < n_worlds; ++k) {
    OWorld* w = static_cast<OWorld*>(handles[k]);
    (w->bodies.size() >= kBigWorld ? big : small).push_back(w);
  }
  std::stable_sort(small.begin(), small.end(), [](OWorld* a, OWorld* b) { return a->bodies.size() > b->bodies.size(); });
  for (OWorld* w : big)
    for (int s = 0; s < steps; ++s) w->step();
  const int ns = (int)small.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt) if (nt > 1 && ns > 1)
  for (int k = 0; k < ns; ++k)
    for (int s = 0; s < steps; ++s) small[k]->step();
}
void orc_world_step(void* h, int n) { OWorld* w = static_cast<OWorld*>(h); for (int s = 0; s < n; ++s) w->step(); }
void orc_world_get_bodies(void* h, exg_body_t* out) {
  OWorld* w = static_cast<OWorld*>(h);
  for (size_t i = 0; i < w->bodies.size(); ++i) from_obody(w->bodies[i], out[i]);
}
// Overwrite every body's pose and momentum (a host moving kinematic bodies between steps, as the
// camera rig's target tracker does in pre_step, crates/hitchcock/src/camera.rs:55-76); the islands
// and their solver state stay.
void orc_world_set_state(void* h, const exg_body_t* bodies) {
  OWorld* w = static_cast<OWorld*>(h);
  for (size_t i = 0; i < w->bodies.size(); ++i) {
    std::memcpy(w->bodies[i].pose, bodies[i].pose, sizeof w->bodies[i].pose);
    std::memcpy(w->bodies[i].mom, bodies[i].momentum, sizeof w->bodies[i].mom);
  }
}
double orc_world_energy(void* h) { return static_cast<OWorld*>(h)->energy(); }
// The epoch of the following steps (Epoch::standalone(dt, warp), crates/aristotle/src/epoch.rs:17-60):
// a host with a variable frame time passes a new dt to every Mechanism::step; the islands stay.
void orc_world_set_epoch(void* h, double dt, double warp) {
  OWorld* w = static_cast<OWorld*>(h);
  w->wp.dt = dt;
  w->wp.warp = warp;
}
// spans / Newton iterations of island k's last step
int orc_world_island_count(void* h) { return (int)static_cast<OWorld*>(h)->islands.size(); }
void orc_world_island_stats(void* h, int k, int* spans, int* iters) {
  Island& isl = static_cast<OWorld*>(h)->islands[k];
  *spans = isl.last_spans;
  *iters = isl.last_newton_iterations;
}

// Structure of island k, in the kinds of exg_world_island_structure (include/exg.h): 1 island
// bodies, 2 joint ends (law, a, b per joint, island-local), 3 order, 4 incidence pointers,
// 5 incidence terms, 7 island joints. Returns the length, or -1 when it exceeds cap.
int orc_world_island_structure(void* h, int k, int kind, int* out, int cap) {
  OWorld* w = static_cast<OWorld*>(h);
  if (!w->built) w->build();
  if (k < 0 || k >= (int)w->islands.size()) return -1;
  const Island& isl = w->islands[k];
  std::vector<int> v, ptr, ref;
  auto local = [&](int g) { return int(std::lower_bound(isl.bodies.begin(), isl.bodies.end(), g) - isl.bodies.begin()); };
  switch (kind) {
    case 1: v = isl.bodies; break;
    case 2:
      for (int jq : isl.joints) {
        const OJoint& j = w->joints[jq];
        v.push_back(j.law); v.push_back(local(j.a)); v.push_back(local(j.b));
      }
      break;
    case 3: v = isl.order; break;
    case 4: bake_incidence(isl, w->joints, ptr, ref); v = ptr; break;
    case 5: bake_incidence(isl, w->joints, ptr, ref); v = ref; break;
    case 7: v = isl.joints; break;
    default: return -1;
  }
  if ((int)v.size() > cap) return -1;
  std::copy(v.begin(), v.end(), out);
  return (int)v.size();
}

// ── stage-level checks ──────────────────────────────────────────────────────
void orc_plain_eval(int law, const double* params, const double* pose_a, const double* pose_b, const double* vel_a,
                    const double* vel_b, double dt, double warp, double* out12) {
  plain_eval(law, params, pose_a, pose_b, vel_a, vel_b, dt, warp, out12);
}
void orc_jacobian_eval(int law, const double* params, const double* pose_a, const double* pose_b, const double* vel_a,
                       const double* vel_b, double dt, double warp, double* out300) {
  jacobian_eval(law, params, pose_a, pose_b, vel_a, vel_b, dt, warp, out300);
}
void orc_gravity_forces(const exg_body_t* bodies, int n, int law, double G, double eps, double* out3) {
  std::vector<OBody> b;
  for (int i = 0; i < n; ++i) b.push_back(to_obody(bodies[i]));
  std::vector<V3<double>> f;
  gravity_forces(b, GravityParams{law, G, eps}, f);
  for (int i = 0; i < n; ++i) for (int k = 0; k < 3; ++k) out3[3 * i + k] = f[i][k];
}
int orc_pair_force_literal(const double* p_lo, double g_lo, const double* p_hi, double g_hi, double size_hi, double* out3) {
  V3<double> f;
  bool ok = pair_force_literal(V3<double>(p_lo[0], p_lo[1], p_lo[2]), g_lo, V3<double>(p_hi[0], p_hi[1], p_hi[2]), g_hi, size_hi, f);
  for (int k = 0; k < 3; ++k) out3[k] = f[k];
  return ok ? 1 : 0;
}
void orc_body_post(const exg_body_t* body, const double* pose_mid, const double* solve_vel, const double* snap_mom,
                   const double* total, double half, double floor2, double* block36, double* rhs6, double* scale6) {
  OBody b = to_obody(*body);
  Block blk;
  body_post(b, Motor<double>::from_components(pose_mid), Twist<double>::from6(solve_vel), Wrench<double>::from6(snap_mom),
            Wrench<double>::from6(total), half, floor2, blk, rhs6, scale6);
  for (int k = 0; k < 36; ++k) block36[k] = blk[k];
}

// ── algebra known-answer helpers ─────────────────────────────────────────────
// Twist::exp(dt) of (linear, angular) -> 8 motor components
void orc_twist_exp(const double* twist6, double dt, double* out8) { twist_exp(Twist<double>::from6(twist6), dt).to_components(out8); }
void orc_motor_compose(const double* a8, const double* b8, double* out8) {
  Motor<double>::from_components(a8).compose(Motor<double>::from_components(b8)).to_components(out8);
}
void orc_motor_inverse(const double* a8, double* out8) { Motor<double>::from_components(a8).inverse().to_components(out8); }
void orc_motor_apply_point(const double* m8, const double* p3, double* out3) {
  Point<double> q = anchor_point(Motor<double>::from_components(m8), V3<double>(p3[0], p3[1], p3[2]));
  V3<double> c = q.coords();
  for (int k = 0; k < 3; ++k) out3[k] = c[k];
}
void orc_twist_transport(const double* t6, const double* m8, int covariant, double* out6) {
  Screw<double> s = Screw<double>::from6(t6);
  Motor<double> m = Motor<double>::from_components(m8);
  (covariant ? s.transport_co(m) : s.transport_contra(m)).to6(out6);
}
double orc_power(const double* w6, const double* t6) { return power(Wrench<double>::from6(w6), Twist<double>::from6(t6)); }
void orc_coad_bracket(const double* w6, const double* t6, double* out6) {
  coad_bracket(Wrench<double>::from6(w6), Twist<double>::from6(t6)).to6(out6);
}
void orc_velocity_at(const double* t6, const double* p3, double* out3) {
  V3<double> v = velocity_at(Twist<double>::from6(t6), Point<double>::at(V3<double>(p3[0], p3[1], p3[2])));
  for (int k = 0; k < 3; ++k) out3[k] = v[k];
}
void orc_study_forms(double u, double* out3) { out3[0] = sinc_sq(u); out3[1] = cos_sq(u); out3[2] = dsinc_sq(u); }
void orc_study_forms_f32(float u, float* out3) { out3[0] = sinc_sq(u); out3[1] = cos_sq(u); out3[2] = dsinc_sq(u); }
// The raw 16-slot blade product sign table, for the sign-law pin tests.
void orc_blade_prod(int a, int b, int* sign, int* mask) { BladeProd p = blade_prod(a, b); *sign = p.sign; *mask = p.mask; }
int orc_angular_embed_sign(void) { return angular_embed_sign(); }
void orc_markup(int kind, int axis, int* mask, int* sign) {
  MaskSign ms = kind == 0 ? euclid_blade(axis) : kind == 1 ? radical_blade(axis) : kind == 2 ? point_blade(axis) : angular_blade(axis);
  *mask = ms.mask; *sign = ms.sign;
}

}  // extern "C"
