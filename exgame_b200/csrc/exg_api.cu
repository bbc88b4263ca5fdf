// C ABI of libexg (include/exg.h): device context, device-resident worlds and the stage calls.
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include "exg_internal.cuh"
#include "body.cuh"
#include "world_newton.cuh"
#include "laws.cuh"
#include "slab.cuh"

namespace {
thread_local std::string g_last_error;
const char* kLawNames[4] = {"SimpleSpringDamper", "CriticallyDampedWarped", "PerpendicularDamperWarped",
                            "TorsionalDamperWarped"};
const int kLawParams[4] = {10, 10, 2, 1};
}  // namespace

void exg_internal_set_message(const char* what) { g_last_error = what; }

void exg_internal_set_cuda_error(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
}

// One admitted world of a pool: its ranges in the pool's arrays and its gravity work items.
struct WorldSlot {
  bool used = false;
  int body_off = 0, n = 0, joint_off = 0, nj = 0;
  long long poff = 0, plen = 0;  // gravity partial range
  int splits = 0;
  std::vector<GravItem> items;   // out_off already relative to the pool's partial array
  exg_step_params_t params{};
};

// A world handle is a pool of worlds: arrays of fixed capacity (bodies, joints, world slots) in
// which worlds are admitted into free ranges and released. A batch is a pool filled once; one
// world is a batch of one. Structural changes mark the handle dirty: the gravity item queue and
// the island queue are rebuilt and the step graph re-captured before the next step.
struct exg_world_s {
  exg_device_s* dev = nullptr;
  std::mutex mu;               // one caller at a time on this handle
  cudaStream_t own = nullptr;  // the handle's own stream (EXG_OPT_OWN_STREAM), else the device's
  DeviceWorld w;
  NewtonWorld* newton = nullptr;
  exg_world_stats_t stats{};
  cudaGraphExec_t graph = nullptr;
  int graph_kernels = 0;
  int b_cap = 0, j_cap = 0, w_cap = 0;
  RangeAllocator body_alloc, joint_alloc, partial_alloc;
  std::vector<WorldSlot> slots;
  int n_explicit = 0, n_implicit = 0, n_used = 0;
  bool dirty = true;
  DevArr<GravItem> items_d;
  DevArr<double> partial_d;
  DevArr<exg_body_t> stage_d;  // host record staging
  DevArr<int> flags_d;         // record check flags (set_records)
  DevArr<int> map_d;           // record -> body of the whole handle's used slots
  bool map_dirty = true;
  std::vector<void*> allocations;

  template <class T> int alloc(T** out, size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    EXG_CUDA_TRY(cudaMalloc(&p, sizeof(T) * count));
    allocations.push_back(p);
    *out = static_cast<T*>(p);
    return EXG_OK;
  }
  void drop_graph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
  ~exg_world_s() {
    drop_graph();
    delete newton;
    items_d.release();
    partial_d.release();
    stage_d.release();
    flags_d.release();
    map_d.release();
    for (void* p : allocations) cudaFree(p);
  }
};

// The stream a handle's work runs on.
static inline cudaStream_t wstream(const exg_world_s* W) { return W->own ? W->own : W->dev->stream; }

// Calls on one handle exclude each other. A handle on the device's stream also excludes every
// other call that uses that stream (a graph captured there must see no foreign work), so only
// handles with their own stream run side by side. Lock order: the handle, then the device.
struct HandleLock {
  std::unique_lock<std::mutex> handle, device;
  explicit HandleLock(exg_world_s* W) : handle(W->mu) {
    if (!W->own) device = std::unique_lock<std::mutex>(W->dev->mu);
  }
};

static cudaEvent_t take_event(exg_device_s* dev) {
  if (!dev->free_events.empty()) {
    cudaEvent_t e = dev->free_events.back();
    dev->free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

int prof_begin(exg_device_s* dev, int kind, cudaStream_t s) {
  if (!dev->profiling) return -1;
  std::lock_guard<std::mutex> lock(dev->prof_mu);
  exg_device_s::Rec r{kind, take_event(dev), take_event(dev)};
  cudaEventRecord(r.a, s);
  dev->recs.push_back(r);
  return (int)dev->recs.size() - 1;
}

void prof_end(exg_device_s* dev, int token, cudaStream_t s) {
  if (token < 0) return;
  std::lock_guard<std::mutex> lock(dev->prof_mu);
  cudaEventRecord(dev->recs[token].b, s);
}

// fold recorded pairs into the per-kind totals (the device must be idle)
static void prof_collect(exg_device_s* dev) {
  std::lock_guard<std::mutex> lock(dev->prof_mu);
  for (auto& r : dev->recs) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      dev->prof_ms[r.kind] += ms;
      dev->prof_count[r.kind] += 1;
    }
    dev->free_events.push_back(r.a);
    dev->free_events.push_back(r.b);
  }
  dev->recs.clear();
}

extern "C" {

int exg_device_stream(exg_device_t dev, void** out) {
  if (!dev || !out) return EXG_ERR_INVALID_ARGUMENT;
  *out = (void*)dev->stream;
  return EXG_OK;
}

int exg_device_profile(exg_device_t dev, int32_t enable) {
  if (!dev) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
  EXG_CUDA_TRY(cudaDeviceSynchronize());  // world handles may run on their own streams
  prof_collect(dev);
  for (int k = 0; k < PROF_KINDS; ++k) { dev->prof_ms[k] = 0.0; dev->prof_count[k] = 0; }
  dev->profiling = enable != 0;
  return EXG_OK;
}

int exg_device_profile_read(exg_device_t dev, int32_t kind, double* total_ms, int64_t* launches) {
  if (!dev || kind < 0 || kind >= PROF_KINDS || !total_ms || !launches) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
  EXG_CUDA_TRY(cudaDeviceSynchronize());
  prof_collect(dev);
  *total_ms = dev->prof_ms[kind];
  *launches = dev->prof_count[kind];
  return EXG_OK;
}

int exg_abi_version(void) { return EXG_ABI_VERSION; }

int exg_device_set_tuning(exg_device_t dev, int32_t key, int32_t value) {
  if (!dev) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  switch (key) {
    case EXG_TUNE_GRAVITY_CTAS_PER_SM:
      if (value < 1 || value > 64) return EXG_ERR_INVALID_ARGUMENT;
      dev->tune_gravity_ctas_per_sm = value;
      return EXG_OK;
    case EXG_TUNE_WAVE_BLOCKS_PER_SM:
      if (value < 1 || value > 32) return EXG_ERR_INVALID_ARGUMENT;
      dev->tune_wave_blocks_per_sm = value;
      return EXG_OK;
    case EXG_TUNE_WAVE_MIN_BODIES:
      if (value < 1) return EXG_ERR_INVALID_ARGUMENT;
      dev->tune_wave_min_bodies = value;
      return EXG_OK;
    case EXG_TUNE_WAVE_NARROW_LEVEL:
      if (value < 1 || value > (1 << 30)) return EXG_ERR_INVALID_ARGUMENT;
      dev->tune_wave_narrow_level = value;
      return EXG_OK;
    default:
      return EXG_ERR_INVALID_ARGUMENT;
  }
}

int exg_device_get_tuning(exg_device_t dev, int32_t key, int32_t* value) {
  if (!dev || !value) return EXG_ERR_INVALID_ARGUMENT;
  switch (key) {
    case EXG_TUNE_GRAVITY_CTAS_PER_SM: *value = dev->tune_gravity_ctas_per_sm; return EXG_OK;
    case EXG_TUNE_WAVE_BLOCKS_PER_SM: *value = dev->tune_wave_blocks_per_sm; return EXG_OK;
    case EXG_TUNE_WAVE_MIN_BODIES: *value = dev->tune_wave_min_bodies; return EXG_OK;
    case EXG_TUNE_WAVE_NARROW_LEVEL: *value = dev->tune_wave_narrow_level; return EXG_OK;
    default: return EXG_ERR_INVALID_ARGUMENT;
  }
}

const char* exg_status_string(int status) {
  switch (status) {
    case EXG_OK: return "ok";
    case EXG_ERR_NO_SHADER: return "no kernel for this joint law";
    case EXG_ERR_TRAP: return "kernel refused its input";
    case EXG_ERR_FATAL: return "a guarded site fired: non-finite state";
    case EXG_ERR_WORKER_GONE: return "the request loop has shut down";
    case EXG_ERR_BACKEND: return g_last_error.empty() ? "CUDA backend error" : g_last_error.c_str();
    case EXG_ERR_EPOCH_IN_PROGRESS: return "structure is frozen while an epoch is in progress";
    case EXG_ERR_ALREADY_OWNED: return "the body already belongs to a mechanism";
    case EXG_ERR_FOREIGN_ACCELERATOR: return "the mechanism runs on a different device";
    case EXG_ERR_DUPLICATE_MECHANISM: return "the mechanism is already registered";
    case EXG_ERR_INVALID_ARGUMENT: return "invalid argument";
    case EXG_ERR_OUT_OF_MEMORY: return "out of device memory";
    case EXG_ERR_UNSUPPORTED: return "unsupported configuration";
    case EXG_ERR_TIMEOUT: return "a bounded wait timed out";
    case EXG_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

int exg_device_create(int32_t ordinal, exg_device_t* out) {
  if (!out) return EXG_ERR_INVALID_ARGUMENT;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return EXG_ERR_NO_DEVICE;
  if (ordinal < 0 || ordinal >= count) return EXG_ERR_INVALID_ARGUMENT;
  exg_device_s* d = new (std::nothrow) exg_device_s();
  if (!d) return EXG_ERR_OUT_OF_MEMORY;
  d->ordinal = ordinal;
  cudaError_t e = cudaSetDevice(ordinal);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d->sm_count, cudaDevAttrMultiProcessorCount, ordinal);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    exg_internal_set_cuda_error(e, "device create");
    delete d;
    return EXG_ERR_BACKEND;
  }
  exg_internal_noalloc_forget(ordinal);
  *out = d;
  return EXG_OK;
}

int exg_device_destroy(exg_device_t dev) {
  if (!dev || dev->handles.load() > 0) return EXG_ERR_INVALID_ARGUMENT;  // its worlds go first
  cudaSetDevice(dev->ordinal);
  cudaStreamSynchronize(dev->stream);
  prof_collect(dev);
  for (cudaEvent_t e : dev->free_events) cudaEventDestroy(e);
  cudaStreamDestroy(dev->stream);
  delete dev;
  return EXG_OK;
}

int exg_device_synchronize(exg_device_t dev) {
  if (!dev) return EXG_ERR_INVALID_ARGUMENT;
  EXG_CUDA_TRY(cudaSetDevice(dev->ordinal));
  EXG_CUDA_TRY(cudaDeviceSynchronize());  // every handle's stream
  return EXG_OK;
}

int exg_device_kernel_launches(exg_device_t dev, uint64_t* out) {
  if (!dev || !out) return EXG_ERR_INVALID_ARGUMENT;
  *out = dev->launches.load();
  return EXG_OK;
}

int exg_law_lookup(const char* name, int32_t* law_out, int32_t* n_params_out) {
  if (!name) return EXG_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 4; ++k)
    if (std::strcmp(name, kLawNames[k]) == 0) {
      if (law_out) *law_out = k;
      if (n_params_out) *n_params_out = kLawParams[k];
      return EXG_OK;
    }
  for (int k = 0; k < exg::kUserLaws; ++k)  // the traced laws (user_laws.cuh)
    if (std::strcmp(name, exg::kUserLawTable[k].name) == 0) {
      if (law_out) *law_out = exg::kUserLawFirst + k;
      if (n_params_out) *n_params_out = exg::kUserLawTable[k].n_params;
      return EXG_OK;
    }
  return EXG_ERR_NO_SHADER;
}

}  // extern "C"

static int validate_world(const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                          const exg_step_params_t* p) {
  if (n < 0 || nj < 0 || (n > 0 && !bodies) || (nj > 0 && !joints) || !p) return EXG_ERR_INVALID_ARGUMENT;
  if (p->integrator < 0 || p->integrator > EXG_NEWTON) return EXG_ERR_INVALID_ARGUMENT;
  if (p->gravity_law < 0 || p->gravity_law > EXG_GRAVITY_PLUMMER) return EXG_ERR_INVALID_ARGUMENT;
  if (p->precision < EXG_PRECISION_F64 || p->precision > EXG_PRECISION_MIXED_FAST) return EXG_ERR_INVALID_ARGUMENT;
  if (p->gravity_law == EXG_GRAVITY_PLUMMER && !(p->softening > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  if (!(p->dt > 0.0) || !(p->warp >= 1.0)) return EXG_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(p->field_accel[k])) return EXG_ERR_INVALID_ARGUMENT;
  for (int32_t i = 0; i < n; ++i)
    if (!bodies[i].kinematic && !(bodies[i].mass > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  for (int32_t k = 0; k < nj; ++k) {
    if (joints[k].law < 0 || joints[k].law >= exg::kUserLawFirst + exg::kUserLaws) return EXG_ERR_NO_SHADER;
    if (joints[k].a < 0 || joints[k].a >= n || joints[k].b < 0 || joints[k].b >= n || joints[k].a == joints[k].b)
      return EXG_ERR_INVALID_ARGUMENT;
  }
  return EXG_OK;
}

// Host records in and out: one copy of the records to (from) a device staging array and one
// kernel between the records and the rows. dst (device, count entries) maps record k to its body;
// null means bodies first .. first + count - 1.
static int stage_reserve(exg_world_s* W, long long count) {
  if (W->stage_d.cap >= count) return EXG_OK;
  W->stage_d.release();  // staging contents never outlive a call
  return W->stage_d.reserve(count, wstream(W));
}

static int upload_records(exg_world_s* W, const exg_body_t* bodies, int32_t first, int32_t count, const int* dst) {
  if (count <= 0) return EXG_OK;
  cudaStream_t s = wstream(W);
  int rc = stage_reserve(W, count);
  if (rc != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaMemcpyAsync(W->stage_d.ptr, bodies, sizeof(exg_body_t) * (size_t)count, cudaMemcpyHostToDevice, s));
  if ((rc = launch_bodies_scatter(W->dev, W->w, W->stage_d.ptr, count, first, dst, s)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

static int download_records(exg_world_s* W, exg_body_t* out, int32_t first, int32_t count, const int* dst) {
  if (count <= 0) return EXG_OK;
  cudaStream_t s = wstream(W);
  int rc = stage_reserve(W, count);
  if (rc != EXG_OK) return rc;
  if ((rc = launch_bodies_gather(W->dev, W->w, W->stage_d.ptr, count, first, dst, s)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaMemcpyAsync(out, W->stage_d.ptr, sizeof(exg_body_t) * (size_t)count, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

// Records that replace bodies of live worlds (exg_world_set_bodies: every used slot in slot order,
// slot < 0; exg_batch_set_world: one slot). The staged records are checked on the device before
// any is written: a dynamic record without positive mass refuses the call, and kinematic flags
// that differ from the current ones rebuild the islands of the implicit worlds they belong to
// (all or none: a structure error restores the worlds already rebuilt).
static int set_records(exg_world_s* W, const exg_body_t* bodies, int32_t first, int32_t count, const int* dst,
                       int slot) {
  if (count <= 0) return EXG_OK;
  cudaStream_t s = wstream(W);
  int rc = stage_reserve(W, count);
  if (rc != EXG_OK) return rc;
  if (W->flags_d.cap < 2 && (rc = W->flags_d.reserve(2, s)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaMemcpyAsync(W->stage_d.ptr, bodies, sizeof(exg_body_t) * (size_t)count, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemsetAsync(W->flags_d.ptr, 0, 2 * sizeof(int), s));
  if ((rc = launch_records_check(W->dev, W->w, W->stage_d.ptr, count, first, dst, W->flags_d.ptr, s)) != EXG_OK)
    return rc;
  int flags[2] = {0, 0};
  EXG_CUDA_TRY(cudaMemcpyAsync(flags, W->flags_d.ptr, sizeof(flags), cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  if (flags[0]) return EXG_ERR_INVALID_ARGUMENT;
  if (flags[1]) {
    std::vector<std::pair<int, std::vector<char>>> done;  // rebuilt slots with their previous flags
    long long k = 0;
    for (int t = 0; t < (int)W->slots.size(); ++t) {
      const WorldSlot& ws = W->slots[t];
      if (!ws.used || (slot >= 0 && t != slot)) continue;
      const exg_body_t* b = bodies + k;
      k += ws.n;
      if (ws.params.integrator != EXG_NEWTON || !W->newton->kin_differs(t, b, ws.n)) continue;
      std::vector<char> kin(ws.n);
      for (int i = 0; i < ws.n; ++i) kin[i] = b[i].kinematic != 0;
      std::vector<char> old = W->newton->kin_of(t);
      if ((rc = W->newton->rebuild_world(t, kin)) != EXG_OK) {
        for (auto& d : done) W->newton->rebuild_world(d.first, d.second);
        return rc;
      }
      done.emplace_back(t, std::move(old));
      W->dirty = true;
    }
  }
  if ((rc = launch_bodies_scatter(W->dev, W->w, W->stage_d.ptr, count, first, dst, s)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

static int upload_bodies(exg_world_s* W, const exg_body_t* bodies, int32_t first, int32_t count) {
  return upload_records(W, bodies, first, count, nullptr);
}

static int download_bodies(exg_world_s* W, exg_body_t* out, int32_t first, int32_t count) {
  return download_records(W, out, first, count, nullptr);
}

// The whole handle's record map: used slots in slot order, each at its body range.
static int ensure_record_map(exg_world_s* W, long long* total) {
  long long n = 0;
  for (auto& ws : W->slots) if (ws.used) n += ws.n;
  *total = n;
  if (!W->map_dirty) return EXG_OK;
  std::vector<int> map;
  map.reserve((size_t)n);
  for (auto& ws : W->slots)
    if (ws.used)
      for (int i = 0; i < ws.n; ++i) map.push_back(ws.body_off + i);
  int rc = W->map_d.assign(map.data(), (long long)map.size(), wstream(W));
  if (rc != EXG_OK) return rc;
  W->map_dirty = false;
  return EXG_OK;
}

static int fill_int(exg_world_s* W, int* d, long long first, long long count, int value) {
  if (count <= 0) return EXG_OK;
  std::vector<int> v(count, value);
  EXG_CUDA_TRY(cudaMemcpyAsync(d + first, v.data(), sizeof(int) * count, cudaMemcpyHostToDevice, wstream(W)));
  EXG_CUDA_TRY(cudaStreamSynchronize(wstream(W)));
  return EXG_OK;
}

template <class T> static int put(exg_world_s* W, T* d, long long first, const T* src, long long count) {
  if (count <= 0) return EXG_OK;
  EXG_CUDA_TRY(cudaMemcpyAsync(d + first, src, sizeof(T) * count, cudaMemcpyHostToDevice, wstream(W)));
  EXG_CUDA_TRY(cudaStreamSynchronize(wstream(W)));
  return EXG_OK;
}

// Allocate a pool's arrays at fixed capacity; every body and joint slot starts unused.
static int pool_init(exg_world_s* W, exg_device_s* dev, int b_cap, int j_cap, int w_cap, int precision) {
  W->dev = dev;
  W->b_cap = b_cap;
  W->j_cap = j_cap;
  W->w_cap = w_cap;
  W->body_alloc.init(b_cap);
  W->joint_alloc.init(j_cap);
  W->partial_alloc.init(0);
  W->slots.resize(w_cap);
  DeviceWorld& w = W->w;
  w.n = b_cap;
  w.nj = j_cap;
  w.n_worlds = w_cap;
  w.precision = precision;
  w.h_params.resize(w_cap);
  w.h_body_off.assign(w_cap, 0);
  w.h_n.assign(w_cap, 0);
  w.h_joint_off.assign(w_cap, 0);
  w.h_nj.assign(w_cap, 0);
  int rc = EXG_OK;
#define ALLOC(ptr, cnt) \
  if (rc == EXG_OK) rc = W->alloc(&(ptr), (cnt))
  ALLOC(w.pose, 8 * (size_t)b_cap);
  ALLOC(w.mom, 6 * (size_t)b_cap);
  ALLOC(w.mass, (size_t)b_cap);
  ALLOC(w.inertia, 9 * (size_t)b_cap);
  ALLOC(w.size, (size_t)b_cap);
  ALLOC(w.kinematic, (size_t)b_cap);
  ALLOC(w.diagonal, (size_t)b_cap);
  ALLOC(w.world_of_body, (size_t)b_cap);
  ALLOC(w.inc_start, (size_t)b_cap);
  ALLOC(w.inc_cnt, (size_t)b_cap);
  ALLOC(w.pos_mass, 4 * (size_t)b_cap);
  ALLOC(w.wvel, 6 * (size_t)b_cap);
  ALLOC(w.joints, (size_t)j_cap);
  ALLOC(w.world_of_joint, (size_t)j_cap);
  ALLOC(w.inc_ref, 2 * (size_t)j_cap);
  ALLOC(w.conn, 12 * (size_t)j_cap);
  ALLOC(w.wparams, (size_t)w_cap);
  ALLOC(w.w_poff, (size_t)w_cap);
  ALLOC(w.w_splits, (size_t)w_cap);
  ALLOC(w.w_n, (size_t)w_cap);
  ALLOC(w.w_body_off, (size_t)w_cap);
  ALLOC(w.w_left, (size_t)w_cap);
  ALLOC(w.w_active, (size_t)w_cap);
  ALLOC(w.item_head, 1);
#undef ALLOC
  if (rc != EXG_OK) return rc;
  cudaStream_t s = dev->stream;
  EXG_CUDA_TRY(cudaMemsetAsync(w.world_of_body, 0xff, sizeof(int) * (size_t)std::max(b_cap, 1), s));
  EXG_CUDA_TRY(cudaMemsetAsync(w.world_of_joint, 0xff, sizeof(int) * (size_t)std::max(j_cap, 1), s));
  EXG_CUDA_TRY(cudaMemsetAsync(w.inc_cnt, 0, sizeof(int) * (size_t)std::max(b_cap, 1), s));
  EXG_CUDA_TRY(cudaMemsetAsync(w.w_active, 0, sizeof(int) * (size_t)std::max(w_cap, 1), s));
  EXG_CUDA_TRY(cudaMemsetAsync(w.w_splits, 0, sizeof(int) * (size_t)std::max(w_cap, 1), s));
  EXG_CUDA_TRY(cudaMemsetAsync(w.w_poff, 0, sizeof(long long) * (size_t)std::max(w_cap, 1), s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  W->newton = new (std::nothrow) NewtonWorld();
  if (!W->newton) return EXG_ERR_OUT_OF_MEMORY;
  W->newton->set_wave_threshold(dev->tune_wave_min_bodies, W->newton->wave_max_levels());
  return EXG_OK;
}

// Admit one validated world into free ranges of the pool.
// A world's joints into the pool's joint range [jo, jo + nj): batch-global body indices, the
// incidence of its n bodies (at bo) in joint order, and the range's owner.
static int upload_joints(exg_world_s* W, int slot, int bo, int n, long long jo, const exg_joint_t* joints, int nj) {
  DeviceWorld& w = W->w;
  std::vector<exg_joint_t> gj(joints, joints + nj);
  for (auto& j : gj) { j.a += bo; j.b += bo; }
  std::vector<int> cnt(n, 0), start(n, 0), ref(2 * (size_t)nj);
  for (int k = 0; k < nj; ++k) { cnt[joints[k].a]++; cnt[joints[k].b]++; }
  int acc = 0;
  for (int i = 0; i < n; ++i) { start[i] = 2 * (int)jo + acc; acc += cnt[i]; }
  std::vector<int> fill(start);
  for (int k = 0; k < nj; ++k) {
    ref[fill[joints[k].a]++ - 2 * jo] = 2 * ((int)jo + k);
    ref[fill[joints[k].b]++ - 2 * jo] = 2 * ((int)jo + k) + 1;
  }
  int rc = put(W, w.joints, jo, gj.data(), nj);
  if (rc == EXG_OK) rc = put(W, w.inc_start, bo, start.data(), n);
  if (rc == EXG_OK) rc = put(W, w.inc_cnt, bo, cnt.data(), n);
  if (rc == EXG_OK) rc = put(W, w.inc_ref, 2 * jo, ref.data(), 2 * (long long)nj);
  if (rc == EXG_OK) rc = fill_int(W, w.world_of_joint, jo, nj, slot);
  return rc;
}

static int pool_admit(exg_world_s* W, const exg_body_t* bodies, int n, const exg_joint_t* joints, int nj,
                      const exg_step_params_t& p, int* slot_out) {
  if (p.precision != W->w.precision) return EXG_ERR_INVALID_ARGUMENT;
  int slot = -1;
  for (int k = 0; k < W->w_cap; ++k)
    if (!W->slots[k].used) { slot = k; break; }
  if (slot < 0) return EXG_ERR_OUT_OF_MEMORY;
  long long bo = W->body_alloc.alloc(n);
  if (bo < 0) return EXG_ERR_OUT_OF_MEMORY;
  long long jo = W->joint_alloc.alloc(nj);
  if (jo < 0) {
    W->body_alloc.release(bo, n);
    return EXG_ERR_OUT_OF_MEMORY;
  }
  DeviceWorld& w = W->w;
  int rc = upload_bodies(W, bodies, (int)bo, n);
  if (rc == EXG_OK) rc = upload_joints(W, slot, (int)bo, n, jo, joints, nj);
  // gravity work items of this world alone (their j-ranges depend on the world's size only)
  WorldSlot ws;
  std::vector<GravItem> items;
  std::vector<int> splits;
  std::vector<long long> poff;
  long long plen = 0;
  gravity_plan({(int)bo}, {n}, {p.gravity_law}, {p.softening}, W->dev->sm_count, items, splits, poff, plen);
  long long po = 0;
  if (plen > 0) {
    po = W->partial_alloc.alloc(plen);
    if (po < 0) {
      long long old = W->partial_alloc.capacity();
      W->partial_alloc.grow(old + std::max(old, plen));
      po = W->partial_alloc.alloc(plen);
    }
  }
  for (auto& g : items) g.out_off += po;
  int sp = splits.empty() ? 0 : splits[0];
  int w_n = n, w_bo = (int)bo, unbounded = -1;
  if (rc == EXG_OK) rc = put(W, w.wparams, slot, &p, 1);
  if (rc == EXG_OK) rc = put(W, w.w_poff, slot, &po, 1);
  if (rc == EXG_OK) rc = put(W, w.w_splits, slot, &sp, 1);
  if (rc == EXG_OK) rc = put(W, w.w_n, slot, &w_n, 1);
  if (rc == EXG_OK) rc = put(W, w.w_body_off, slot, &w_bo, 1);
  if (rc == EXG_OK) rc = put(W, w.w_left, slot, &unbounded, 1);
  if (rc == EXG_OK && p.integrator == EXG_NEWTON) rc = W->newton->add_world(W->dev, slot, (int)bo, bodies, n, joints, nj);
  if (rc == EXG_OK) rc = fill_int(W, w.world_of_body, bo, n, slot);  // last: the world becomes visible
  if (rc != EXG_OK) {
    fill_int(W, w.world_of_joint, jo, nj, -1);
    W->body_alloc.release(bo, n);
    W->joint_alloc.release(jo, nj);
    if (plen > 0) W->partial_alloc.release(po, plen);
    return rc;
  }
  ws.used = true;
  ws.body_off = (int)bo;
  ws.n = n;
  ws.joint_off = (int)jo;
  ws.nj = nj;
  ws.poff = po;
  ws.plen = plen;
  ws.splits = sp;
  ws.items = std::move(items);
  ws.params = p;
  W->slots[slot] = std::move(ws);
  w.h_params[slot] = p;
  w.h_body_off[slot] = (int)bo;
  w.h_n[slot] = n;
  w.h_joint_off[slot] = (int)jo;
  w.h_nj[slot] = nj;
  if (p.integrator == EXG_NEWTON) ++W->n_implicit; else ++W->n_explicit;
  ++W->n_used;
  W->dirty = true;
  W->map_dirty = true;
  *slot_out = slot;
  return EXG_OK;
}

static int pool_release(exg_world_s* W, int slot) {
  if (slot < 0 || slot >= W->w_cap || !W->slots[slot].used) return EXG_ERR_INVALID_ARGUMENT;
  WorldSlot& ws = W->slots[slot];
  int rc = fill_int(W, W->w.world_of_body, ws.body_off, ws.n, -1);
  if (rc == EXG_OK) rc = fill_int(W, W->w.world_of_joint, ws.joint_off, ws.nj, -1);
  int zero = 0;
  if (rc == EXG_OK) rc = put(W, W->w.w_splits, slot, &zero, 1);
  if (rc != EXG_OK) return rc;
  if (ws.params.integrator == EXG_NEWTON) { W->newton->remove_world(slot); --W->n_implicit; } else --W->n_explicit;
  W->body_alloc.release(ws.body_off, ws.n);
  W->joint_alloc.release(ws.joint_off, ws.nj);
  if (ws.plen > 0) W->partial_alloc.release(ws.poff, ws.plen);
  ws = WorldSlot();
  --W->n_used;
  W->dirty = true;
  W->map_dirty = true;
  return EXG_OK;
}

// New joints for the world in `slot` (Islands::connect / detach and Mechanism::split / merge as
// one edit: the islands are the connected components of the new joint graph, rebuilt on the
// host). Its bodies stay on the device. All or nothing: a refused structure, or no room in the
// joint range, leaves the world as it was.
static int pool_set_joints(exg_world_s* W, int slot, const exg_joint_t* joints, int nj) {
  WorldSlot& ws = W->slots[slot];
  for (int k = 0; k < nj; ++k) {
    if (joints[k].law < 0 || joints[k].law >= exg::kUserLawFirst + exg::kUserLaws) return EXG_ERR_NO_SHADER;
    if (joints[k].a < 0 || joints[k].a >= ws.n || joints[k].b < 0 || joints[k].b >= ws.n || joints[k].a == joints[k].b)
      return EXG_ERR_INVALID_ARGUMENT;
  }
  long long jo = W->joint_alloc.alloc(nj);
  bool reused = false;  // no room beside the old list: its range is given up first
  if (jo < 0) {
    W->joint_alloc.release(ws.joint_off, ws.nj);
    reused = true;
    jo = W->joint_alloc.alloc(nj);
    if (jo < 0) {
      W->joint_alloc.alloc_at(ws.joint_off, ws.nj);  // just released: free
      return EXG_ERR_OUT_OF_MEMORY;
    }
  }
  int rc = EXG_OK;
  if (ws.params.integrator == EXG_NEWTON && (rc = W->newton->replace_joints(slot, joints, nj)) != EXG_OK) {
    W->joint_alloc.release(jo, nj);
    if (reused) W->joint_alloc.alloc_at(ws.joint_off, ws.nj);
    return rc;
  }
  if ((rc = fill_int(W, W->w.world_of_joint, ws.joint_off, ws.nj, -1)) != EXG_OK) return rc;
  if ((rc = upload_joints(W, slot, ws.body_off, ws.n, jo, joints, nj)) != EXG_OK) return rc;
  if (!reused) W->joint_alloc.release(ws.joint_off, ws.nj);
  ws.joint_off = (int)jo;
  ws.nj = nj;
  W->w.h_joint_off[slot] = (int)jo;
  W->w.h_nj[slot] = nj;
  W->dirty = true;
  return EXG_OK;
}

// Before a step after a structural change: the gravity queue of the live worlds (largest item
// first), the partial array's size, the island queue; the step graph is re-captured.
static int pool_prepare(exg_world_s* W) {
  if (!W->dirty) return EXG_OK;
  W->drop_graph();
  DeviceWorld& w = W->w;
  cudaStream_t s = wstream(W);
  std::vector<std::pair<double, GravItem>> tmp;
  for (auto& ws : W->slots)
    if (ws.used)
      for (auto& g : ws.items) tmp.push_back({double(std::min(kGravTile, g.n - g.i0)) * (g.j1 - g.j0), g});
  std::stable_sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<GravItem> items;
  items.reserve(tmp.size());
  for (auto& x : tmp) items.push_back(x.second);
  int rc = W->items_d.assign(items.data(), (long long)items.size(), s);
  if (rc != EXG_OK) return rc;
  if (W->partial_d.cap < W->partial_alloc.capacity()) {
    W->partial_d.release();  // per-step contents: no copy needed
    if ((rc = W->partial_d.reserve(std::max<long long>(W->partial_alloc.capacity(), 1), s)) != EXG_OK) return rc;
  }
  w.items = W->items_d.ptr;
  w.n_items = (int)items.size();
  w.grav_partial = W->partial_d.ptr;
  w.n_ext = (int)W->body_alloc.used_end();
  w.nj_ext = (int)W->joint_alloc.used_end();
  w.any_explicit = W->n_explicit > 0;
  w.any_newton = W->n_implicit > 0;
  if ((rc = W->newton->sync(W->dev, s)) != EXG_OK) return rc;
  W->dirty = false;
  return EXG_OK;
}

extern "C" {

int exg_batch_create(exg_device_t dev, int32_t n_worlds, const int32_t* body_counts, const int32_t* joint_counts,
                     const exg_body_t* bodies, const exg_joint_t* joints, const exg_step_params_t* params,
                     exg_world_t* out) {
  if (!dev || !out || n_worlds <= 0 || !body_counts || !joint_counts || !params) return EXG_ERR_INVALID_ARGUMENT;
  long long n_total = 0, nj_total = 0;
  for (int32_t wi = 0; wi < n_worlds; ++wi) {
    if (body_counts[wi] < 0 || joint_counts[wi] < 0) return EXG_ERR_INVALID_ARGUMENT;
    int st = validate_world(bodies + n_total, body_counts[wi], joints + nj_total, joint_counts[wi], params + wi);
    if (st != EXG_OK) return st;
    if (params[wi].precision != params[0].precision) return EXG_ERR_INVALID_ARGUMENT;
    n_total += body_counts[wi];
    nj_total += joint_counts[wi];
  }
  if (n_total > (1LL << 30) || nj_total > (1LL << 29)) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
  exg_world_s* W = new (std::nothrow) exg_world_s();
  if (!W) return EXG_ERR_OUT_OF_MEMORY;
  int rc = pool_init(W, dev, (int)n_total, (int)nj_total, n_worlds, params[0].precision);
  long long bo = 0, jo = 0;
  for (int32_t wi = 0; wi < n_worlds && rc == EXG_OK; ++wi) {
    int slot = -1;
    rc = pool_admit(W, bodies + bo, body_counts[wi], joints + jo, joint_counts[wi], params[wi], &slot);
    bo += body_counts[wi];
    jo += joint_counts[wi];
  }
  if (rc == EXG_OK) rc = pool_prepare(W);
  if (rc != EXG_OK) { delete W; return rc; }
  ++dev->handles;
  *out = W;
  return EXG_OK;
}

int exg_world_create(exg_device_t dev, const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                     const exg_step_params_t* params, exg_world_t* out) {
  return exg_batch_create(dev, 1, &n, &nj, bodies, joints, params, out);
}

int exg_pool_create(exg_device_t dev, const exg_pool_config_t* cfg, exg_world_t* out) {
  if (!dev || !cfg || !out || cfg->max_bodies <= 0 || cfg->max_joints < 0 || cfg->max_worlds <= 0) return EXG_ERR_INVALID_ARGUMENT;
  if (cfg->precision < EXG_PRECISION_F64 || cfg->precision > EXG_PRECISION_MIXED_FAST) return EXG_ERR_INVALID_ARGUMENT;
  if (cfg->max_bodies > (1LL << 30) || cfg->max_joints > (1LL << 29)) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
  exg_world_s* W = new (std::nothrow) exg_world_s();
  if (!W) return EXG_ERR_OUT_OF_MEMORY;
  int rc = pool_init(W, dev, (int)cfg->max_bodies, (int)cfg->max_joints, cfg->max_worlds, cfg->precision);
  if (rc != EXG_OK) { delete W; return rc; }
  ++dev->handles;
  *out = W;
  return EXG_OK;
}

int exg_pool_admit(exg_world_t W, const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                   const exg_step_params_t* params, int32_t* slot_out) {
  if (!W || !slot_out) return EXG_ERR_INVALID_ARGUMENT;
  int st = validate_world(bodies, n, joints, nj, params);
  if (st != EXG_OK) return st;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  int slot = -1;
  int rc = pool_admit(W, bodies, n, joints, nj, *params, &slot);
  if (rc == EXG_OK) *slot_out = slot;
  return rc;
}

int exg_pool_release(exg_world_t W, int32_t slot) {
  if (!W) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  return pool_release(W, slot);
}

int exg_pool_free(exg_world_t W, exg_pool_usage_t* out) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  out->worlds_used = W->n_used;
  out->worlds_capacity = W->w_cap;
  out->largest_free_bodies = W->body_alloc.largest_free();
  out->largest_free_joints = W->joint_alloc.largest_free();
  return EXG_OK;
}

int exg_host_alloc(size_t bytes, void** out) {
  if (!out || bytes == 0) return EXG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  EXG_CUDA_TRY(cudaMallocHost(out, bytes));
  return EXG_OK;
}

int exg_host_free(void* p) {
  if (!p) return EXG_ERR_INVALID_ARGUMENT;
  EXG_CUDA_TRY(cudaFreeHost(p));
  return EXG_OK;
}

int exg_world_footprint(int32_t n, int32_t nj, const exg_step_params_t* p, int64_t* bytes) {
  if (!p || !bytes || n < 0 || nj < 0) return EXG_ERR_INVALID_ARGUMENT;
  // pool rows: pose 8, momentum 6, mass, inertia 9, size, charge 4, world twist 6 doubles; kinematic,
  // diagonal, world, incidence start and count ints. Joints: the record, its world, two incidence
  // references and the 12 wrench components.
  long long b = (long long)n * ((8 + 6 + 1 + 9 + 1 + 4 + 6) * 8 + 5 * 4) +
                (long long)nj * ((long long)sizeof(exg_joint_t) + 3 * 4 + 12 * 8);
  if (p->gravity_law != EXG_GRAVITY_OFF && n > 1) {
    int L = kGravTile;
    while (L < 2048 && L * 8 < n) L *= 2;
    long long splits = (n + L - 1) / L, itiles = (n + kGravTile - 1) / kGravTile;
    b += splits * 3 * (long long)n * 8 + splits * itiles * (long long)sizeof(GravItem);
  }
  if (p->integrator == EXG_NEWTON) b += newton_footprint_bytes(n, nj);
  *bytes = b;
  return EXG_OK;
}

int exg_pool_set_steps(exg_world_t W, int32_t slot, int32_t steps) {
  if (!W || slot < 0 || slot >= W->w_cap || !W->slots[slot].used || steps < -1) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  return put(W, W->w.w_left, slot, &steps, 1);
}

int exg_pool_steps_left(exg_world_t W, int32_t* out, int32_t n_slots) {
  if (!W || !out || n_slots < 0 || n_slots > W->w_cap) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  if (n_slots == 0) return EXG_OK;
  EXG_CUDA_TRY(cudaMemcpyAsync(out, W->w.w_left, sizeof(int32_t) * n_slots, cudaMemcpyDeviceToHost, wstream(W)));
  EXG_CUDA_TRY(cudaStreamSynchronize(wstream(W)));
  for (int32_t k = 0; k < n_slots; ++k)
    if (!W->slots[k].used) out[k] = 0;
  return EXG_OK;
}

int exg_world_set_option(exg_world_t W, int32_t option, int64_t value) {
  if (!W) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  switch (option) {
    case EXG_OPT_WAVE_MIN_BODIES:
      if (value < 1 || value > (1LL << 30)) return EXG_ERR_INVALID_ARGUMENT;
      W->newton->set_wave_threshold((int)value, W->newton->wave_max_levels());
      break;
    case EXG_OPT_WAVE_MAX_LEVELS:
      if (value < 1 || value > (1LL << 30)) return EXG_ERR_INVALID_ARGUMENT;
      W->newton->set_wave_threshold(W->newton->wave_min_dyn(), (int)value);
      break;
    case EXG_OPT_WAVE_HOST_ROUNDS:
      if (value != 0 && value != 1) return EXG_ERR_INVALID_ARGUMENT;
      W->newton->set_wave_host_loop(value != 0);
      return EXG_OK;
    case EXG_OPT_OWN_STREAM:
      if (value != 0 && value != 1) return EXG_ERR_INVALID_ARGUMENT;
      EXG_CUDA_TRY(cudaSetDevice(W->dev->ordinal));
      EXG_CUDA_TRY(cudaStreamSynchronize(wstream(W)));  // work in flight ends where it began
      if (value && !W->own) {
        EXG_CUDA_TRY(cudaStreamCreateWithFlags(&W->own, cudaStreamNonBlocking));
      } else if (!value && W->own) {
        cudaStreamDestroy(W->own);
        W->own = nullptr;
      }
      return EXG_OK;
    default:
      return EXG_ERR_INVALID_ARGUMENT;
  }
  W->dirty = true;
  return EXG_OK;
}

int exg_world_stream(exg_world_t W, void** out) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  *out = (void*)wstream(W);
  return EXG_OK;
}

int exg_world_get_option(exg_world_t W, int32_t option, int64_t* value) {
  if (!W || !value) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  switch (option) {
    case EXG_OPT_WAVE_MIN_BODIES: *value = W->newton->wave_min_dyn(); return EXG_OK;
    case EXG_OPT_WAVE_MAX_LEVELS: *value = W->newton->wave_max_levels(); return EXG_OK;
    case EXG_OPT_LAST_WAVE_ROUNDS: *value = W->newton->last_wave_rounds(); return EXG_OK;
    case EXG_OPT_WAVE_HOST_ROUNDS: *value = W->newton->wave_host_loop() ? 1 : 0; return EXG_OK;
    case EXG_OPT_OWN_STREAM: *value = W->own ? 1 : 0; return EXG_OK;
    case EXG_OPT_WAVE_LEVEL_MAX_WIDTH: *value = W->newton->wave_level_width(true); return EXG_OK;
    case EXG_OPT_WAVE_LEVEL_MIN_WIDTH: *value = W->newton->wave_level_width(false); return EXG_OK;
    default: return EXG_ERR_INVALID_ARGUMENT;
  }
}

int exg_world_destroy(exg_world_t W) {
  if (!W) return EXG_ERR_INVALID_ARGUMENT;
  exg_device_s* dev = W->dev;
  {
    HandleLock lock(W);  // waits for a call in flight on the handle
    cudaSetDevice(dev->ordinal);
    cudaStreamSynchronize(wstream(W));
  }
  if (W->own) cudaStreamDestroy(W->own);
  delete W;
  --dev->handles;
  return EXG_OK;
}

}  // extern "C"

// One step of every live world (Mechanism::step per world, all enqueued asynchronously):
// charges and world twists, gravity, explicit joints and integration, then the implicit islands.
static int enqueue_step(exg_world_s* W, int* kernels) {
  DeviceWorld& w = W->w;
  cudaStream_t s = wstream(W);
  uint64_t before = W->dev->launches.load();
  int rc;
  if ((rc = launch_body_pre(W->dev, w, s)) != EXG_OK) return rc;
  if ((rc = launch_gravity_items(W->dev, w.pos_mass, w.size, w.items, w.n_items, w.item_head, w.precision,
                                 w.grav_partial, s, w.world_of_body, w.w_active)) != EXG_OK)
    return rc;
  if ((rc = launch_joints_plain_world(W->dev, w, s)) != EXG_OK) return rc;
  if ((rc = launch_integrate_explicit(W->dev, w, s)) != EXG_OK) return rc;
  if ((rc = W->newton->enqueue(W->dev, w, s)) != EXG_OK) return rc;
  *kernels = (int)(W->dev->launches.load() - before);
  return EXG_OK;
}

static int step_locked(exg_world_s* W, int32_t n_steps) {
  cudaStream_t s = wstream(W);
  int rc = pool_prepare(W);
  if (rc != EXG_OK) return rc;
  if (W->n_used == 0 || n_steps == 0) return EXG_OK;
  if (W->dev->profiling) {
    for (int32_t k = 0; k < n_steps; ++k) {
      int kernels = 0;
      rc = enqueue_step(W, &kernels);
      if (rc == EXG_OK && W->newton->has_wave()) rc = W->newton->run_wave(W->dev, W->w, s);
      if (rc != EXG_OK) return rc;
    }
  } else {
    if (!W->graph) {
      // capture one step; replays skip the per-launch host cost
      cudaGraph_t g;
      EXG_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int kernels = 0;
      uint64_t before = W->dev->launches.load();
      rc = enqueue_step(W, &kernels);
      W->dev->launches.store(before);  // captured, not yet launched
      cudaError_t e = cudaStreamEndCapture(s, &g);
      if (rc != EXG_OK) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        return rc;
      }
      EXG_CUDA_TRY(e);
      cudaError_t ie = cudaGraphInstantiate(&W->graph, g, 0);
      cudaGraphDestroy(g);
      EXG_CUDA_TRY(ie);
      W->graph_kernels = kernels;
    }
    for (int32_t k = 0; k < n_steps; ++k) {
      EXG_CUDA_TRY(cudaGraphLaunch(W->graph, s));
      W->dev->launches.fetch_add(W->graph_kernels);
      // large islands: the wave schedule's rounds, after the step's other kernels
      if (W->newton->has_wave() && (rc = W->newton->run_wave(W->dev, W->w, s)) != EXG_OK) return rc;
    }
  }
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  if (W->newton->has_wave() && (rc = W->newton->wave_after_steps(W->dev)) != EXG_OK) return rc;
  W->stats.steps += n_steps;
  W->stats.last_spans = 1;
  if (W->n_implicit > 0) {
    rc = W->newton->read_stats(-1, &W->stats);
    if (rc != EXG_OK) return rc;
    if (W->stats.fatal) return EXG_ERR_FATAL;
  }
  return EXG_OK;
}

extern "C" {

int exg_world_step(exg_world_t W, int32_t n_steps) {
  if (!W || n_steps < 0) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  return step_locked(W, n_steps);
}

// whole-handle accessors: the used worlds in slot order, each at its body offset
int exg_world_get_bodies(exg_world_t W, exg_body_t* out, int32_t n) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  long long total = 0;
  int rc = ensure_record_map(W, &total);
  if (rc != EXG_OK) return rc;
  if (n != total) return EXG_ERR_INVALID_ARGUMENT;
  return download_records(W, out, 0, n, W->map_d.ptr);
}

int exg_world_get_state(exg_world_t W, double* out, int32_t n) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  long long total = 0;
  int rc = ensure_record_map(W, &total);
  if (rc != EXG_OK) return rc;
  if (n != total) return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  if ((rc = stage_reserve(W, n)) != EXG_OK) return rc;  // 14 doubles fit in a record's slot
  cudaStream_t s = wstream(W);
  double* st = reinterpret_cast<double*>(W->stage_d.ptr);
  if ((rc = launch_state_gather(W->dev, W->w, st, n, 0, W->map_d.ptr, s)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaMemcpyAsync(out, st, sizeof(double) * 14 * (size_t)n, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

int exg_world_set_state(exg_world_t W, const double* state, int32_t n) {
  if (!W || !state) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  long long total = 0;
  int rc = ensure_record_map(W, &total);
  if (rc != EXG_OK) return rc;
  if (n != total) return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  if ((rc = stage_reserve(W, n)) != EXG_OK) return rc;
  cudaStream_t s = wstream(W);
  double* st = reinterpret_cast<double*>(W->stage_d.ptr);
  EXG_CUDA_TRY(cudaMemcpyAsync(st, state, sizeof(double) * 14 * (size_t)n, cudaMemcpyHostToDevice, s));
  if ((rc = launch_state_scatter(W->dev, W->w, st, n, 0, W->map_d.ptr, s)) != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

int exg_world_set_bodies(exg_world_t W, const exg_body_t* bodies, int32_t n) {
  if (!W || !bodies) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  long long total = 0;
  int rc = ensure_record_map(W, &total);
  if (rc != EXG_OK) return rc;
  if (n != total) return EXG_ERR_INVALID_ARGUMENT;
  return set_records(W, bodies, 0, n, W->map_d.ptr, -1);
}

int exg_batch_get_world(exg_world_t W, int32_t world, exg_body_t* out, int32_t n) {
  if (!W || !out || world < 0 || world >= W->w_cap || !W->slots[world].used || n != W->slots[world].n)
    return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  return download_bodies(W, out, W->slots[world].body_off, n);
}

int exg_batch_set_joints(exg_world_t W, int32_t world, const exg_joint_t* joints, int32_t nj) {
  if (!W || world < 0 || world >= W->w_cap || !W->slots[world].used || nj < 0 || (nj > 0 && !joints))
    return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  return pool_set_joints(W, world, joints, nj);
}

int exg_batch_set_world(exg_world_t W, int32_t world, const exg_body_t* bodies, int32_t n) {
  if (!W || !bodies || world < 0 || world >= W->w_cap || !W->slots[world].used || n != W->slots[world].n)
    return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  return set_records(W, bodies, W->slots[world].body_off, n, nullptr, world);
}

int exg_world_stats(exg_world_t W, exg_world_stats_t* out) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  *out = W->stats;
  return EXG_OK;
}

int exg_batch_world_stats(exg_world_t W, int32_t world, exg_world_stats_t* out) {
  if (!W || !out || world < 0 || world >= W->w_cap || !W->slots[world].used) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  *out = W->stats;
  out->last_spans = 1;
  out->last_newton_iterations = 0;
  out->max_depth_reached = 0;
  out->fatal = 0;
  out->last_residual = 0.0;
  if (W->slots[world].params.integrator == EXG_NEWTON) return W->newton->read_stats(world, out);
  return EXG_OK;
}

int exg_world_phase_cycles(exg_world_t W, int64_t out[8]) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  cudaSetDevice(W->dev->ordinal);
  long long tmp[8];
  int rc = W->newton->read_phase_cycles(tmp);
  for (int k = 0; k < 8; ++k) out[k] = tmp[k];
  return rc;
}

int exg_batch_set_epoch(exg_world_t W, int32_t world, double dt, double warp) {
  if (!W || !(dt > 0.0) || !std::isfinite(dt) || !(warp >= 1.0) || !std::isfinite(warp)) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  if (world < 0 || world >= W->w_cap || !W->slots[world].used) return EXG_ERR_INVALID_ARGUMENT;
  EXG_CUDA_TRY(cudaSetDevice(W->dev->ordinal));
  exg_step_params_t p = W->slots[world].params;
  p.dt = dt;
  p.warp = warp;
  int rc = put(W, W->w.wparams, world, &p, 1);
  if (rc != EXG_OK) return rc;
  W->slots[world].params = p;
  W->w.h_params[world] = p;
  return EXG_OK;
}

int exg_world_island_count(exg_world_t W, int32_t world, int32_t* n_islands) {
  if (!W || !n_islands) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  if (world < 0 || world >= W->w_cap || !W->slots[world].used) return EXG_ERR_INVALID_ARGUMENT;
  *n_islands = W->newton->island_count(world);
  return EXG_OK;
}

int exg_world_island_structure(exg_world_t W, int32_t world, int32_t island, int32_t kind, int32_t* out, int32_t cap,
                               int32_t* len) {
  if (!W || !len || cap < 0 || (cap > 0 && !out)) return EXG_ERR_INVALID_ARGUMENT;
  HandleLock lock(W);
  if (world < 0 || world >= W->w_cap || !W->slots[world].used) return EXG_ERR_INVALID_ARGUMENT;
  EXG_CUDA_TRY(cudaSetDevice(W->dev->ordinal));
  int rc;
  if (W->dirty && (rc = pool_prepare(W)) != EXG_OK) return rc;  // upload pending structure first
  int n = 0;
  rc = W->newton->read_structure(world, island, kind, out, cap, &n);
  *len = n;
  return rc;
}

int exg_world_energy(exg_world_t W, double* out) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  double e = 0.0;
  for (int k = 0; k < W->w_cap; ++k) {
    const WorldSlot& ws = W->slots[k];
    if (!ws.used) continue;
    std::vector<exg_body_t> b(ws.n);
    int rc = exg_batch_get_world(W, k, b.data(), ws.n);
    if (rc != EXG_OK) return rc;
    std::vector<exg_joint_t> j(ws.nj);
    if (ws.nj > 0) {
      HandleLock lock(W);
      EXG_CUDA_TRY(cudaMemcpy(j.data(), W->w.joints + ws.joint_off, sizeof(exg_joint_t) * ws.nj, cudaMemcpyDeviceToHost));
    }
    for (auto& jj : j) { jj.a -= ws.body_off; jj.b -= ws.body_off; }
    e += host_world_energy(b.data(), ws.n, j.data(), ws.nj, ws.params);
  }
  *out = e;
  return EXG_OK;
}

int exg_motor_exp(const double twist[6], double dt, double out[8]) {
  if (!twist || !out) return EXG_ERR_INVALID_ARGUMENT;
  double b[6];
  exg::screw_from6(twist, b);
  exg::twist_exp(b, dt, out);
  return EXG_OK;
}
int exg_motor_exp_n(int64_t count, const double* twists, double dt, double* out) {
  if (count < 0 || (count > 0 && (!twists || !out))) return EXG_ERR_INVALID_ARGUMENT;
  for (int64_t k = 0; k < count; ++k) {
    double b[6];
    exg::screw_from6(twists + 6 * k, b);
    exg::twist_exp(b, dt, out + 8 * k);
  }
  return EXG_OK;
}
int exg_motor_compose_n(int64_t count, const double* a, const double* b, double* out) {
  if (count < 0 || (count > 0 && (!a || !b || !out))) return EXG_ERR_INVALID_ARGUMENT;
  for (int64_t k = 0; k < count; ++k) {
    double r[8];
    exg::motor_compose(a + 8 * k, b + 8 * k, r);
    for (int c = 0; c < 8; ++c) out[8 * k + c] = r[c];
  }
  return EXG_OK;
}
int exg_motor_compose(const double a[8], const double b[8], double out[8]) {
  if (!a || !b || !out) return EXG_ERR_INVALID_ARGUMENT;
  double r[8];
  exg::motor_compose(a, b, r);
  for (int k = 0; k < 8; ++k) out[k] = r[k];
  return EXG_OK;
}
int exg_motor_inverse(const double a[8], double out[8]) {
  if (!a || !out) return EXG_ERR_INVALID_ARGUMENT;
  double r[8];
  exg::motor_reverse(a, r);
  for (int k = 0; k < 8; ++k) out[k] = r[k];
  return EXG_OK;
}
int exg_motor_apply_point(const double m[8], const double p[3], double out[3]) {
  if (!m || !p || !out) return EXG_ERR_INVALID_ARGUMENT;
  double q[4];
  exg::anchor_point(m, p, q);
  exg::point_coords(q, out);
  return EXG_OK;
}
int exg_screw_transport(const double s6[6], const double m[8], int32_t covariant, double out[6]) {
  if (!s6 || !m || !out) return EXG_ERR_INVALID_ARGUMENT;
  double b[6], r[6];
  exg::screw_from6(s6, b);
  if (covariant) exg::wrench_transport(b, m, r); else exg::twist_transport(b, m, r);
  exg::screw_to6(r, out);
  return EXG_OK;
}

int exg_eval_joints(exg_device_t dev, const exg_joint_t* d_joints, int32_t nj, const double* d_pose, const double* d_vel,
                    double dt, double warp, int32_t jacobian, double* d_out) {
  if (!dev || nj < 0 || (nj > 0 && (!d_joints || !d_pose || !d_vel || !d_out))) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(dev->ordinal));
  int rc = launch_joints_stage(dev, d_joints, nj, d_pose, d_vel, dt, warp, jacobian, d_out, dev->stream);
  if (rc != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(dev->stream));
  return EXG_OK;
}

int exg_pivot_inverse(exg_device_t dev, const double* d_blocks, int32_t n, int32_t precision, int32_t form,
                      int32_t warm, double* d_out, int32_t* d_steps) {
  if (!dev || n < 0 || (n > 0 && (!d_blocks || !d_out))) return EXG_ERR_INVALID_ARGUMENT;
  if (precision != EXG_PRECISION_F64 && precision != EXG_PRECISION_MIXED && precision != EXG_PRECISION_MIXED_FAST)
    return EXG_ERR_INVALID_ARGUMENT;
  if (form != 0 && form != 1) return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  std::lock_guard<std::mutex> lock(dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(dev->ordinal));
  cudaStream_t s = dev->stream;
  int* d_singular = nullptr;
  EXG_CUDA_TRY(cudaMallocAsync(&d_singular, sizeof(int), s));
  int rc = EXG_OK;
  if (cudaMemsetAsync(d_singular, 0, sizeof(int), s) != cudaSuccess) rc = EXG_ERR_BACKEND;
  if (rc == EXG_OK)
    rc = launch_pivot_inverse(dev, d_blocks, n, precision != EXG_PRECISION_F64, form, warm, d_out, d_steps, d_singular,
                              s);
  int h_singular = 0;
  if (rc == EXG_OK && cudaMemcpyAsync(&h_singular, d_singular, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    rc = EXG_ERR_BACKEND;
  cudaFreeAsync(d_singular, s);
  if (rc != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return h_singular ? EXG_ERR_FATAL : EXG_OK;
}

int exg_gravity_forces(exg_device_t dev, const double* d_pos_mass, const double* d_size, int32_t n, int32_t law, double G,
                       double softening, int32_t precision, double* d_force) {
  if (!dev || n < 0 || (n > 0 && (!d_pos_mass || !d_force))) return EXG_ERR_INVALID_ARGUMENT;
  if (law == EXG_GRAVITY_SIZE_CORE && n > 0 && !d_size) return EXG_ERR_INVALID_ARGUMENT;
  if (law != EXG_GRAVITY_SIZE_CORE && law != EXG_GRAVITY_PLUMMER) return EXG_ERR_INVALID_ARGUMENT;
  if (law == EXG_GRAVITY_PLUMMER && !(softening > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  if (precision != EXG_PRECISION_F64 && precision != EXG_PRECISION_MIXED && precision != EXG_PRECISION_MIXED_FAST)
    return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  std::lock_guard<std::mutex> lock(dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(dev->ordinal));
  cudaStream_t s = dev->stream;
  if (n == 1) {
    EXG_CUDA_TRY(cudaMemsetAsync(d_force, 0, 3 * sizeof(double), s));
    EXG_CUDA_TRY(cudaStreamSynchronize(s));
    return EXG_OK;
  }
  std::vector<GravItem> items;
  std::vector<int> splits;
  std::vector<long long> poff;
  long long plen = 0;
  gravity_plan({0}, {n}, {law}, {softening}, dev->sm_count, items, splits, poff, plen);
  double* partial = nullptr;
  GravItem* d_items = nullptr;
  int* head = nullptr;
  EXG_CUDA_TRY(cudaMallocAsync(&partial, sizeof(double) * plen, s));
  EXG_CUDA_TRY(cudaMallocAsync(&d_items, sizeof(GravItem) * items.size(), s));
  EXG_CUDA_TRY(cudaMallocAsync(&head, sizeof(int), s));
  EXG_CUDA_TRY(cudaMemcpyAsync(d_items, items.data(), sizeof(GravItem) * items.size(), cudaMemcpyHostToDevice, s));
  int rc = launch_gravity_items(dev, d_pos_mass, d_size, d_items, (int)items.size(), head, precision, partial, s);
  if (rc == EXG_OK) rc = launch_gravity_reduce(dev, partial, d_pos_mass, n, splits[0], G, d_force, s);
  cudaFreeAsync(partial, s);
  cudaFreeAsync(d_items, s);
  cudaFreeAsync(head, s);
  if (rc != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

}  // extern "C"
