// Internal definitions shared by the translation units of libexg: the device context, the
// device-resident batch of worlds (structure-of-arrays), error plumbing and the launch wrappers
// each .cu file provides.
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
// The message exg_status_string(EXG_ERR_BACKEND) returns on this thread until the next error.
void exg_internal_set_message(const char* what);
// One-writer check of a scatter map (storage.cu): every entry of slots[0, n) in [0, n_slots) and no
// slot named twice. EXG_OK, or EXG_ERR_BACKEND with the message set and *first_clash the position
// of the first repeated (or out-of-range) entry.
int exg_internal_ledger(const int32_t* slots, long long n, long long n_slots, long long* first_clash, const char* what);
// Drop the cached device address of the no-allocation gravity array on `ordinal` (gravity.cu).
void exg_internal_noalloc_forget(int ordinal);

// Kernel kinds the in-library profiler distinguishes.
enum ProfKind { PROF_GRAVITY = 0, PROF_JOINTS = 1, PROF_INTEGRATE = 2, PROF_NEWTON = 3, PROF_BODY_PRE = 4, PROF_NEWTON_WAVE = 5,
                PROF_KINDS = 8 };

struct exg_device_s {
  int ordinal = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  std::atomic<uint64_t> launches{0};
  std::mutex mu;  // one submitter at a time (the reference's single worker thread)
  std::atomic<int> handles{0};  // live world handles made on the device (batches, pools, servers' pools)
  // profiler: event pairs recorded on `stream` around each launch of a kind
  std::atomic<bool> profiling{false};
  std::mutex prof_mu;  // the event records below (handles on their own streams record concurrently)
  struct Rec { int kind; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> free_events;
  double prof_ms[PROF_KINDS] = {0};
  long long prof_count[PROF_KINDS] = {0};
  // launch-shape tuning (exg_device_set_tuning; results do not depend on any of these)
  std::atomic<int> tune_gravity_ctas_per_sm{32};  // persistent one-warp CTAs of the mixed gravity kernel
  std::atomic<int> tune_wave_blocks_per_sm{16};   // grid cap of the wave's 256-thread data kernels (128-thread: twice)
  std::atomic<int> tune_wave_min_bodies{32};      // default wave threshold of new world handles
  std::atomic<int> tune_wave_narrow_level{8192};  // elimination levels up to this many nodes: a warp per node
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

// One unit of gravity work: an i-tile of one world's bodies against a j-range of the same world.
// The partial sum  sum_j m_j r_ij / core^3  of body (body_off + i) lands at
// partial[out_off + c * n + (i - 0)] for component c.
struct GravItem {
  int body_off;   // first body of the world (global index)
  int n;          // bodies in the world
  int i0;         // first i (world-local) of the tile
  int j0, j1;     // world-local j range
  int law;        // EXG_GRAVITY_SIZE_CORE or EXG_GRAVITY_PLUMMER
  double eps2;    // Plummer softening squared
  long long out_off;
};
constexpr int kGravTile = 128;

// Build the gravity work items of a set of worlds (descending work, so the persistent kernel
// schedules longest-first). Returns the per-world split count and partial offset.
void gravity_plan(const std::vector<int>& body_off, const std::vector<int>& n, const std::vector<int>& law,
                  const std::vector<double>& eps, int sm_count, std::vector<GravItem>& items,
                  std::vector<int>& splits, std::vector<long long>& poff, long long& partial_len);

// Device-resident batch of worlds. Per-body quantities are component-major over all bodies of
// the batch: component c of body i at [c*n + i].
struct DeviceWorld {
  int n = 0, nj = 0, n_worlds = 0, precision = 0;  // n, nj: array strides (capacities)
  int n_ext = 0, nj_ext = 0;  // bodies / joints below which every used slot lies (launch extents)
  double* pose = nullptr;      // [8][n]
  double* mom = nullptr;       // [6][n] body-frame momentum
  double* mass = nullptr;      // [n]
  double* inertia = nullptr;   // [9][n]
  double* size = nullptr;      // [n]
  int* kinematic = nullptr;    // [n]
  int* diagonal = nullptr;     // [n]
  int* world_of_body = nullptr;     // [n], -1 for an unused slot
  exg_joint_t* joints = nullptr;    // [nj], body indices global to the batch
  int* world_of_joint = nullptr;    // [nj], -1 for an unused slot
  int* inc_start = nullptr;    // [n] first incident joint end of each body in inc_ref
  int* inc_cnt = nullptr;      // [n] number of incident joint ends
  int* inc_ref = nullptr;      // [2*nj] joint*2 + end, per body in joint order
  // per world
  exg_step_params_t* wparams = nullptr;  // [n_worlds]
  long long* w_poff = nullptr;           // gravity partial offset per world
  int* w_splits = nullptr;               // gravity splits per world (0: no gravity)
  int* w_n = nullptr;                    // bodies per world
  int* w_body_off = nullptr;             // first body of each world
  int* w_left = nullptr;                 // steps the world still takes (-1: unbounded)
  int* w_active = nullptr;               // 1 when the world takes the current step
  // gravity work items and the persistent scheduler's counter
  GravItem* items = nullptr;
  int n_items = 0;
  int* item_head = nullptr;
  // per-step scratch
  double* pos_mass = nullptr;      // [n] x,y,z,m (double4)
  double* wvel = nullptr;          // [6][n] world twist (lin, ang)
  double* grav_partial = nullptr;  // per world [splits][3][n_w]
  double* conn = nullptr;          // [12][nj]
  bool any_explicit = false, any_newton = false;
  // host mirrors
  std::vector<exg_step_params_t> h_params;
  std::vector<int> h_body_off, h_n, h_joint_off, h_nj;
};

// ── launch wrappers (each returns an exg_status) ─────────────────────────────
int launch_body_pre(exg_device_s* dev, const DeviceWorld& w, cudaStream_t s);
int launch_gravity_items(exg_device_s* dev, const double* pos_mass, const double* size, const GravItem* items, int n_items,
                         int* head, int precision, double* partial, cudaStream_t s,
                         const int* world_of_body = nullptr, const int* w_active = nullptr);
int launch_gravity_reduce(exg_device_s* dev, const double* partial, const double* pos_mass, int n, int splits, double G,
                          double* force_out, cudaStream_t s);
int launch_joints_plain_world(exg_device_s* dev, const DeviceWorld& w, cudaStream_t s);
int launch_joints_stage(exg_device_s* dev, const exg_joint_t* joints, int nj, const double* pose_aos, const double* vel_aos,
                        double dt, double warp, int jacobian, double* out, cudaStream_t s);
int launch_integrate_explicit(exg_device_s* dev, const DeviceWorld& w, cudaStream_t s);
// the elimination's pivot inverse on n row-major 6x6 blocks: mixed != 0 the Newton-Schulz inverse
// (warm != 0: out holds earlier inverses to start from), else FP64 Gauss-Jordan; form 0 one thread
// per block, 1 one warp
int launch_pivot_inverse(exg_device_s* dev, const double* blocks, int n, int mixed, int form, int warm, double* out,
                         int* steps, int* singular, cudaStream_t s);
// records <-> rows: record k is body first + k, or body dst[k] when dst is not null
int launch_bodies_scatter(exg_device_s* dev, const DeviceWorld& w, const exg_body_t* rec, int count, int first,
                          const int* dst, cudaStream_t s);
int launch_state_scatter(exg_device_s* dev, const DeviceWorld& w, const double* st, int count, int first,
                         const int* dst, cudaStream_t s);
int launch_state_gather(exg_device_s* dev, const DeviceWorld& w, double* st, int count, int first, const int* dst,
                        cudaStream_t s);
int launch_records_check(exg_device_s* dev, const DeviceWorld& w, const exg_body_t* rec, int count, int first,
                         const int* dst, int* flags, cudaStream_t s);
int launch_bodies_gather(exg_device_s* dev, const DeviceWorld& w, exg_body_t* rec, int count, int first,
                         const int* dst, cudaStream_t s);
