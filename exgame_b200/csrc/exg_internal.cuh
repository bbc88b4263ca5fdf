// Internal definitions shared by the translation units of libexg: the device context, the
// device-resident world (structure-of-arrays), error plumbing and the launch wrappers each
// .cu file provides.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <mutex>
#include <vector>
#include "../../include/exg.h"

#define EXG_CUDA_TRY(expr)                          \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) {                        \
      exg_internal_set_cuda_error(_e, #expr);       \
      return EXG_ERR_BACKEND;                       \
    }                                               \
  } while (0)

void exg_internal_set_cuda_error(cudaError_t e, const char* what);

// Kernel kinds the in-library profiler distinguishes.
enum ProfKind { PROF_GRAVITY = 0, PROF_JOINTS = 1, PROF_INTEGRATE = 2, PROF_NEWTON = 3, PROF_BODY_PRE = 4, PROF_KINDS = 8 };

struct exg_device_s {
  int ordinal = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  std::atomic<uint64_t> launches{0};
  std::mutex mu;  // one submitter at a time (the reference's single worker thread)
  // profiler: event pairs recorded on `stream` around each launch of a kind
  bool profiling = false;
  struct Rec { int kind; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> free_events;
  double prof_ms[PROF_KINDS] = {0};
  long long prof_count[PROF_KINDS] = {0};
};

// Brackets one launch with events when profiling is on (no-op otherwise).
int prof_begin(exg_device_s* dev, int kind, cudaStream_t s);
void prof_end(exg_device_s* dev, int token, cudaStream_t s);

// Count one kernel launch on the device and check the launch status.
inline int exg_after_launch(exg_device_s* dev) {
  dev->launches.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { exg_internal_set_cuda_error(e, "kernel launch"); return EXG_ERR_BACKEND; }
  return EXG_OK;
}

// Gravity launch shape: i-tile width (threads per CTA) and the number of j-splits whose
// partial forces are summed in a fixed order afterwards (deterministic, no atomics).
struct GravityShape { int tile; int splits; };
GravityShape gravity_pick_shape(int n, int sm_count, int precision);

// World storage. Per-body quantities are stored component-major: comp c of body i at [c*n + i].
struct DeviceWorld {
  int n = 0, nj = 0;
  double* pose = nullptr;      // [8][n]
  double* mom = nullptr;       // [6][n] body-frame momentum
  double* mass = nullptr;      // [n]
  double* inertia = nullptr;   // [9][n]
  double* size = nullptr;      // [n]
  int* kinematic = nullptr;    // [n]
  int* diagonal = nullptr;     // [n]
  exg_joint_t* joints = nullptr;  // [nj]
  int* inc_ptr = nullptr;      // [n+1] body -> incident joint ends (CSR)
  int* inc_ref = nullptr;      // [2*nj] joint*2 + end, in joint order
  // per-step scratch
  double* pos_mass = nullptr;  // [n] x,y,z,m (double4)
  double* wvel = nullptr;      // [6][n] world twist (lin, ang)
  double* grav_partial = nullptr;  // [splits][3][n]
  double* conn = nullptr;      // [12][nj]
  int grav_splits = 1;
  GravityShape gshape{64, 1};
};

// ── launch wrappers (each returns an exg_status) ─────────────────────────────
int launch_body_pre(exg_device_s* dev, const DeviceWorld& w, cudaStream_t s);
int launch_gravity(exg_device_s* dev, const double* pos_mass, const double* size, int n, int law, double softening,
                   int precision, GravityShape shape, double* partial, cudaStream_t s);
int launch_gravity_reduce(exg_device_s* dev, const double* partial, const double* pos_mass, int n, int splits, double G,
                          double* force_out, cudaStream_t s);
int launch_joints_plain_world(exg_device_s* dev, const DeviceWorld& w, double dt, double warp, cudaStream_t s);
int launch_joints_stage(exg_device_s* dev, const exg_joint_t* joints, int nj, const double* pose_aos, const double* vel_aos,
                        double dt, double warp, int jacobian, double* out, cudaStream_t s);
int launch_integrate_explicit(exg_device_s* dev, const DeviceWorld& w, int scheme, int gravity_on, double G, double dt,
                              cudaStream_t s);
