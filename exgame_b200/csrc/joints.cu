// Joint kernels K1-K8 (crates/newton/build.rs:874-973): one thread per joint for the plain
// value kernel; one thread per (joint, 6-axis slice) for the Jacobian kernel, the four slices
// of a joint being adjacent threads of one warp.
#include "exg_internal.cuh"
#include "joint_eval.cuh"

namespace {

// World form: poses [8][n] and world twists [6][n] component-major; output conn[12][nj]. Joints
// of worlds stepped by the implicit integrator are evaluated inside the Newton kernel instead.
__global__ void k_joints_plain_world(const exg_joint_t* __restrict__ joints, const int* __restrict__ world_of_joint,
                                     const int* __restrict__ w_active, const exg_step_params_t* __restrict__ wparams, int nj,
                                     const double* __restrict__ pose, const double* __restrict__ wvel, int n,
                                     double* __restrict__ conn) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nj) return;
  const int wid = world_of_joint[k];
  if (wid < 0 || !w_active[wid]) return;
  const exg_step_params_t& P = wparams[wid];
  if (P.integrator == EXG_NEWTON) return;
  const exg_joint_t& jt = joints[k];
  double pa[8], pb[8], va[6], vb[6], out[12];
#pragma unroll
  for (int c = 0; c < 8; ++c) { pa[c] = pose[(size_t)c * n + jt.a]; pb[c] = pose[(size_t)c * n + jt.b]; }
#pragma unroll
  for (int c = 0; c < 6; ++c) { va[c] = wvel[(size_t)c * n + jt.a]; vb[c] = wvel[(size_t)c * n + jt.b]; }
  exg::joint_plain<double>(jt.law, jt.params, pa, pb, va, vb, P.dt, P.warp, out);
#pragma unroll
  for (int c = 0; c < 12; ++c) conn[(size_t)c * nj + k] = out[c];
}

// Stage form: poses [body][8], twists [body][6] (AoS); plain out[k][12] or Jacobian out[k][300].
__global__ void k_joints_stage_plain(const exg_joint_t* __restrict__ joints, int nj, const double* __restrict__ pose,
                                     const double* __restrict__ vel, double dt, double warp, double* __restrict__ out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nj) return;
  const exg_joint_t& jt = joints[k];
  exg::joint_plain<double>(jt.law, jt.params, pose + 8 * (size_t)jt.a, pose + 8 * (size_t)jt.b, vel + 6 * (size_t)jt.a,
                           vel + 6 * (size_t)jt.b, dt, warp, out + 12 * (size_t)k);
}

__global__ void k_joints_stage_jacobian(const exg_joint_t* __restrict__ joints, int nj, const double* __restrict__ pose,
                                        const double* __restrict__ vel, double dt, double warp, double* __restrict__ out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int k = t >> 2, slice = t & 3;
  if (k >= nj) return;
  const exg_joint_t& jt = joints[k];
  double pa[8], pb[8], va[6], vb[6];
#pragma unroll
  for (int c = 0; c < 8; ++c) { pa[c] = pose[8 * (size_t)jt.a + c]; pb[c] = pose[8 * (size_t)jt.b + c]; }
#pragma unroll
  for (int c = 0; c < 6; ++c) { va[c] = vel[6 * (size_t)jt.a + c]; vb[c] = vel[6 * (size_t)jt.b + c]; }
  double v[6], d[36];
  exg::joint_jacobian_slice<double>(jt.law, jt.params, pa, pb, va, vb, dt, warp, slice, v, d);
  double* o = out + 300 * (size_t)k;
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    if (slice == 0) { o[r * 25] = v[r]; o[(6 + r) * 25] = -v[r]; }
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      o[r * 25 + 1 + 6 * slice + c] = d[r * 6 + c];
      o[(6 + r) * 25 + 1 + 6 * slice + c] = -d[r * 6 + c];
    }
  }
}

}  // namespace

int launch_joints_plain_world(exg_device_s* dev, const DeviceWorld& w, cudaStream_t s) {
  if (w.nj_ext <= 0 || !w.any_explicit) return EXG_OK;
  int _tok = prof_begin(dev, PROF_JOINTS, s);
  k_joints_plain_world<<<(w.nj_ext + 127) / 128, 128, 0, s>>>(w.joints, w.world_of_joint, w.w_active, w.wparams, w.nj, w.pose, w.wvel,
                                                          w.n, w.conn);
  prof_end(dev, _tok, s);
  return exg_after_launch(dev);
}

int launch_joints_stage(exg_device_s* dev, const exg_joint_t* joints, int nj, const double* pose_aos, const double* vel_aos,
                        double dt, double warp, int jacobian, double* out, cudaStream_t s) {
  if (nj <= 0) return EXG_OK;
  int _tok = prof_begin(dev, PROF_JOINTS, s);
  if (jacobian) {
    long threads = 4L * nj;
    k_joints_stage_jacobian<<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(joints, nj, pose_aos, vel_aos, dt, warp, out);
  } else {
    k_joints_stage_plain<<<(nj + 127) / 128, 128, 0, s>>>(joints, nj, pose_aos, vel_aos, dt, warp, out);
  }
  prof_end(dev, _tok, s);
  return exg_after_launch(dev);
}
