// Per-body kernels of the explicit step (crates/newton/src/integrator/implicit/bridge.rs:19-63):
//   k_body_pre:          position + mass (gravity charge) and world twist of every body;
//   k_integrate_explicit: gather of the world wrench (gravity + incident joint wrenches in the
//                        reference's term order), pull-back to the body frame and one step of
//                        ExplicitEuler / SymplecticEuler / LieEuler (integrator/explicit/*.rs).
// Poses and momenta stay FP64 in every precision mode.
#include "exg_internal.cuh"
#include "body.cuh"

namespace {

using namespace exg;

// The thread of a world's first body also decides whether the world takes this step (its step
// budget is not spent) and spends one step of it; every later kernel of the step reads w_active.
__global__ void k_body_pre(BodyView b, const int* __restrict__ world_of_body, const int* __restrict__ w_body_off,
                           int* __restrict__ w_left, int* __restrict__ w_active, double* __restrict__ pos_mass,
                           double* __restrict__ wvel) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.n) return;
  const int wid = world_of_body[i];
  if (wid < 0) return;
  if (w_body_off[wid] == i) {
    const int left = w_left[wid];
    w_active[wid] = left != 0;
    if (left > 0) w_left[wid] = left - 1;
  }
  double pose[8], mom[6], I9[9];
  load_body(b, i, pose, mom, I9);
  bool kin = b.kinematic[i] != 0;
  double p3[3];
  body_position(pose, p3);
  double4 pm = make_double4(p3[0], p3[1], p3[2], kin ? 0.0 : b.mass[i]);
  reinterpret_cast<double4*>(pos_mass)[i] = pm;
  double wv[6];
  world_velocity(pose, mom, I9, b.diagonal[i] != 0, kin, b.mass[i], wv);
#pragma unroll
  for (int c = 0; c < 6; ++c) wvel[(size_t)c * b.n + i] = wv[c];
}

// One explicit step of every body whose world uses an explicit scheme; the scheme, dt, G and the
// gravity partial layout come from the body's world.
__global__ void k_integrate_explicit(BodyView b, double* __restrict__ pose_out, double* __restrict__ mom_out,
                                     const double* __restrict__ pos_mass, const double* __restrict__ grav_partial,
                                     const int* __restrict__ world_of_body, const exg_step_params_t* __restrict__ wparams,
                                     const long long* __restrict__ w_poff, const int* __restrict__ w_splits,
                                     const int* __restrict__ w_n, const int* __restrict__ w_body_off,
                                     const int* __restrict__ w_active, const double* __restrict__ conn, int nj, const int* __restrict__ inc_start,
                                     const int* __restrict__ inc_cnt, const int* __restrict__ inc_ref) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.n) return;
  const int wid = world_of_body[i];
  if (wid < 0 || b.kinematic[i] || !w_active[wid]) return;
  const int scheme = wparams[wid].integrator;
  if (scheme == EXG_NEWTON) return;
  const double dt = wparams[wid].dt;
  double pose[8], mom[6], I9[9];
  load_body(b, i, pose, mom, I9);
  const bool diag = b.diagonal[i] != 0;
  const double mass = b.mass[i];
  // world wrench: gravity (F, p x F) then incident joint wrenches in joint order
  double tot[6] = {0, 0, 0, 0, 0, 0};
  const int splits = w_splits[wid];
  if (splits > 0) {
    double4 pm = reinterpret_cast<const double4*>(pos_mass)[i];
    const int nw = w_n[wid];
    const int il = i - w_body_off[wid];
    const double* part = grav_partial + w_poff[wid];
    double f[3];
    for (int c = 0; c < 3; ++c) {
      double acc = 0.0;
      for (int s = 0; s < splits; ++s) acc += part[(size_t)s * 3 * nw + (size_t)c * nw + il];
      f[c] = wparams[wid].G * pm.w * acc;
    }
    tot[0] = f[0]; tot[1] = f[1]; tot[2] = f[2];
    tot[3] = pm.y * f[2] - pm.z * f[1];
    tot[4] = pm.z * f[0] - pm.x * f[2];
    tot[5] = pm.x * f[1] - pm.y * f[0];
  }
  add_uniform_field(wparams[wid].field_accel, reinterpret_cast<const double4*>(pos_mass)[i], tot);
  for (int q = inc_start[i], qe = inc_start[i] + inc_cnt[i]; q < qe; ++q) {
    int ref = inc_ref[q];
    int k = ref >> 1, end = ref & 1;
#pragma unroll
    for (int c = 0; c < 6; ++c) tot[c] += conn[(size_t)(end * 6 + c) * nj + k];
  }
  // pull back to the body frame: transport(pose^-1) under the Co law
  double wb[6], wbody[6], rev[8], tmp[6];
  screw_from6(tot, wb);
  motor_reverse(pose, rev);
  wrench_transport(wb, rev, tmp);
  screw_to6(tmp, wbody);
  if (scheme == EXG_LIE_EULER) {  // lie_euler.rs:31-55
#pragma unroll
    for (int c = 0; c < 6; ++c) mom[c] += wbody[c] * dt;
    double v6[6], vb[6], delta[8], drot[8], drot_inv[8], mb[6], mt[6];
    inertia_inverse(I9, diag, false, mass, mom, v6);
    screw_from6(v6, vb);
    twist_exp(vb, dt, delta);
    motor_rotation_part(delta, drot);
    motor_reverse(drot, drot_inv);
    screw_from6(mom, mb);
    wrench_transport(mb, drot_inv, mt);
    screw_to6(mt, mom);
    double np[8];
    motor_compose(delta, pose, np);  // pose * delta
#pragma unroll
    for (int c = 0; c < 8; ++c) pose[c] = np[c];
  } else {
    double v6[6], vb[6], mb[6], gy[6], gyro[6];
    inertia_inverse(I9, diag, false, mass, mom, v6);
    screw_from6(v6, vb);
    screw_from6(mom, mb);
    coad_bracket(mb, vb, gy);
    screw_to6(gy, gyro);  // gyroscopic = -coad_bracket (body.rs:170-175)
#pragma unroll
    for (int c = 0; c < 6; ++c) mom[c] += (wbody[c] - gyro[c]) * dt;
    if (scheme == EXG_SYMPLECTIC_EULER) {  // symplectic_euler.rs:26-41: the pose moves with the NEW velocity
      inertia_inverse(I9, diag, false, mass, mom, v6);
      screw_from6(v6, vb);
    }  // explicit_euler.rs:21-33: the pose moves with the OLD velocity
    double e[8], np[8];
    twist_exp(vb, dt, e);
    motor_compose(e, pose, np);  // pose * exp
#pragma unroll
    for (int c = 0; c < 8; ++c) pose[c] = np[c];
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) pose_out[(size_t)c * b.n + i] = pose[c];
#pragma unroll
  for (int c = 0; c < 6; ++c) mom_out[(size_t)c * b.n + i] = mom[c];
}

// Host records <-> the pool's component-major rows. Record k belongs to body first + k, or to
// body dst[k] when a map is given (the whole handle's used slots in slot order).
__global__ void k_bodies_scatter(const exg_body_t* __restrict__ rec, int count, int first, const int* __restrict__ dst,
                                 double* pose, double* mom, double* mass, double* inertia, double* size, int* kin,
                                 int* diag, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const exg_body_t& r = rec[k];
  const int i = dst ? dst[k] : first + k;
#pragma unroll
  for (int c = 0; c < 8; ++c) pose[(size_t)c * n + i] = r.pose[c];
#pragma unroll
  for (int c = 0; c < 6; ++c) mom[(size_t)c * n + i] = r.momentum[c];
#pragma unroll
  for (int c = 0; c < 9; ++c) inertia[(size_t)c * n + i] = r.inertia[c];
  mass[i] = r.mass;
  size[i] = r.size;
  kin[i] = r.kinematic;
  diag[i] = r.diagonal;
}

// Dynamic state only — per body pose[8] then momentum[6], the first 14 doubles of a record — and
// the pool's rows. Record k belongs to body first + k, or to body dst[k] when a map is given.
__global__ void k_state_scatter(const double* __restrict__ st, int count, int first, const int* __restrict__ dst,
                                double* pose, double* mom, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const double2* r = reinterpret_cast<const double2*>(st + 14 * (size_t)k);
  double v[14];
#pragma unroll
  for (int e = 0; e < 7; ++e) { const double2 x = r[e]; v[2 * e] = x.x; v[2 * e + 1] = x.y; }
  const int i = dst ? dst[k] : first + k;
#pragma unroll
  for (int c = 0; c < 8; ++c) pose[(size_t)c * n + i] = v[c];
#pragma unroll
  for (int c = 0; c < 6; ++c) mom[(size_t)c * n + i] = v[8 + c];
}

__global__ void k_state_gather(double* __restrict__ st, int count, int first, const int* __restrict__ dst,
                               const double* pose, const double* mom, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int i = dst ? dst[k] : first + k;
  double v[14];
#pragma unroll
  for (int c = 0; c < 8; ++c) v[c] = pose[(size_t)c * n + i];
#pragma unroll
  for (int c = 0; c < 6; ++c) v[8 + c] = mom[(size_t)c * n + i];
  double2* r = reinterpret_cast<double2*>(st + 14 * (size_t)k);
#pragma unroll
  for (int e = 0; e < 7; ++e) r[e] = make_double2(v[2 * e], v[2 * e + 1]);
}

// Records staged for exg_world_set_bodies / exg_batch_set_world, checked before any is written:
// flags[0] = some dynamic record has no positive mass (the call is refused), flags[1] = some
// record's kinematic flag differs from its body's current one (implicit worlds rebuild islands).
__global__ void k_records_check(const exg_body_t* __restrict__ rec, int count, int first, const int* __restrict__ dst,
                                const int* __restrict__ kin, int* flags) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false, changed = false;
  if (k < count) {
    const exg_body_t& r = rec[k];
    const int i = dst ? dst[k] : first + k;
    bad = !r.kinematic && !(r.mass > 0.0);
    changed = (r.kinematic != 0) != (kin[i] != 0);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags, 1);
  if (__syncthreads_or(changed) && threadIdx.x == 0) atomicOr(flags + 1, 1);
}

__global__ void k_bodies_gather(exg_body_t* __restrict__ rec, int count, int first, const int* __restrict__ dst,
                                const double* pose, const double* mom, const double* mass, const double* inertia,
                                const double* size, const int* kin, const int* diag, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  exg_body_t& r = rec[k];
  const int i = dst ? dst[k] : first + k;
#pragma unroll
  for (int c = 0; c < 8; ++c) r.pose[c] = pose[(size_t)c * n + i];
#pragma unroll
  for (int c = 0; c < 6; ++c) r.momentum[c] = mom[(size_t)c * n + i];
#pragma unroll
  for (int c = 0; c < 9; ++c) r.inertia[c] = inertia[(size_t)c * n + i];
  r.mass = mass[i];
  r.size = size[i];
  r.kinematic = kin[i];
  r.diagonal = diag[i];
}

BodyView view_of(const DeviceWorld& w) {
  return BodyView{w.pose, w.mom, w.mass, w.inertia, w.kinematic, w.diagonal, w.n};
}

}  // namespace

int launch_body_pre(exg_device_s* dev, const DeviceWorld& w, cudaStream_t s) {
  if (w.n_ext <= 0) return EXG_OK;
  int _tok = prof_begin(dev, PROF_BODY_PRE, s);
  k_body_pre<<<(w.n_ext + 127) / 128, 128, 0, s>>>(view_of(w), w.world_of_body, w.w_body_off, w.w_left, w.w_active,
                                               w.pos_mass, w.wvel);
  prof_end(dev, _tok, s);
  return exg_after_launch(dev);
}

int launch_integrate_explicit(exg_device_s* dev, const DeviceWorld& w, cudaStream_t s) {
  if (w.n_ext <= 0 || !w.any_explicit) return EXG_OK;
  int tok = prof_begin(dev, PROF_INTEGRATE, s);
  k_integrate_explicit<<<(w.n_ext + 127) / 128, 128, 0, s>>>(view_of(w), w.pose, w.mom, w.pos_mass, w.grav_partial,
                                                         w.world_of_body, w.wparams, w.w_poff, w.w_splits, w.w_n,
                                                         w.w_body_off, w.w_active, w.conn, w.nj, w.inc_start, w.inc_cnt,
                                                         w.inc_ref);
  prof_end(dev, tok, s);
  return exg_after_launch(dev);
}

int launch_bodies_scatter(exg_device_s* dev, const DeviceWorld& w, const exg_body_t* rec, int count, int first,
                          const int* dst, cudaStream_t s) {
  if (count <= 0) return EXG_OK;
  k_bodies_scatter<<<(count + 127) / 128, 128, 0, s>>>(rec, count, first, dst, w.pose, w.mom, w.mass, w.inertia, w.size,
                                                       w.kinematic, w.diagonal, w.n);
  return exg_after_launch(dev);
}

int launch_state_scatter(exg_device_s* dev, const DeviceWorld& w, const double* st, int count, int first,
                         const int* dst, cudaStream_t s) {
  if (count <= 0) return EXG_OK;
  k_state_scatter<<<(count + 127) / 128, 128, 0, s>>>(st, count, first, dst, w.pose, w.mom, w.n);
  return exg_after_launch(dev);
}

int launch_state_gather(exg_device_s* dev, const DeviceWorld& w, double* st, int count, int first, const int* dst,
                        cudaStream_t s) {
  if (count <= 0) return EXG_OK;
  k_state_gather<<<(count + 127) / 128, 128, 0, s>>>(st, count, first, dst, w.pose, w.mom, w.n);
  return exg_after_launch(dev);
}

int launch_records_check(exg_device_s* dev, const DeviceWorld& w, const exg_body_t* rec, int count, int first,
                         const int* dst, int* flags, cudaStream_t s) {
  if (count <= 0) return EXG_OK;
  k_records_check<<<(count + 255) / 256, 256, 0, s>>>(rec, count, first, dst, w.kinematic, flags);
  return exg_after_launch(dev);
}

int launch_bodies_gather(exg_device_s* dev, const DeviceWorld& w, exg_body_t* rec, int count, int first,
                         const int* dst, cudaStream_t s) {
  if (count <= 0) return EXG_OK;
  k_bodies_gather<<<(count + 127) / 128, 128, 0, s>>>(rec, count, first, dst, w.pose, w.mom, w.mass, w.inertia, w.size,
                                                      w.kinematic, w.diagonal, w.n);
  return exg_after_launch(dev);
}
