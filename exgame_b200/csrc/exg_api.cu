// C ABI of libexg (include/exg.h): device context, device-resident worlds and the stage calls.
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include "exg_internal.cuh"
#include "body.cuh"
#include "world_newton.cuh"

namespace {
thread_local std::string g_last_error;
const char* kLawNames[4] = {"SimpleSpringDamper", "CriticallyDampedWarped", "PerpendicularDamperWarped",
                            "TorsionalDamperWarped"};
const int kLawParams[4] = {10, 10, 2, 1};
}  // namespace

void exg_internal_set_cuda_error(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
}

struct exg_world_s {
  exg_device_s* dev = nullptr;
  exg_step_params_t p{};
  DeviceWorld w;
  NewtonWorld* newton = nullptr;
  exg_world_stats_t stats{};
  cudaGraphExec_t graph = nullptr;
  int graph_kernels = 0;
  std::vector<void*> allocations;

  template <class T> int alloc(T** out, size_t count) {
    if (count == 0) count = 1;
    void* p = nullptr;
    EXG_CUDA_TRY(cudaMalloc(&p, sizeof(T) * count));
    allocations.push_back(p);
    *out = static_cast<T*>(p);
    return EXG_OK;
  }
  ~exg_world_s() {
    if (graph) cudaGraphExecDestroy(graph);
    delete newton;
    for (void* p : allocations) cudaFree(p);
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
  exg_device_s::Rec r{kind, take_event(dev), take_event(dev)};
  cudaEventRecord(r.a, s);
  dev->recs.push_back(r);
  return (int)dev->recs.size() - 1;
}

void prof_end(exg_device_s* dev, int token, cudaStream_t s) {
  if (token < 0) return;
  cudaEventRecord(dev->recs[token].b, s);
}

// fold recorded pairs into the per-kind totals (the stream must be idle)
static void prof_collect(exg_device_s* dev) {
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
  EXG_CUDA_TRY(cudaStreamSynchronize(dev->stream));
  prof_collect(dev);
  for (int k = 0; k < PROF_KINDS; ++k) { dev->prof_ms[k] = 0.0; dev->prof_count[k] = 0; }
  dev->profiling = enable != 0;
  return EXG_OK;
}

int exg_device_profile_read(exg_device_t dev, int32_t kind, double* total_ms, int64_t* launches) {
  if (!dev || kind < 0 || kind >= PROF_KINDS || !total_ms || !launches) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
  EXG_CUDA_TRY(cudaStreamSynchronize(dev->stream));
  prof_collect(dev);
  *total_ms = dev->prof_ms[kind];
  *launches = dev->prof_count[kind];
  return EXG_OK;
}

int exg_abi_version(void) { return EXG_ABI_VERSION; }

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
  *out = d;
  return EXG_OK;
}

int exg_device_destroy(exg_device_t dev) {
  if (!dev) return EXG_ERR_INVALID_ARGUMENT;
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
  EXG_CUDA_TRY(cudaStreamSynchronize(dev->stream));
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
  return EXG_ERR_NO_SHADER;
}

}  // extern "C"

static int validate_world(const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                          const exg_step_params_t* p) {
  if (n < 0 || nj < 0 || (n > 0 && !bodies) || (nj > 0 && !joints) || !p) return EXG_ERR_INVALID_ARGUMENT;
  if (p->integrator < 0 || p->integrator > EXG_NEWTON) return EXG_ERR_INVALID_ARGUMENT;
  if (p->gravity_law < 0 || p->gravity_law > EXG_GRAVITY_PLUMMER) return EXG_ERR_INVALID_ARGUMENT;
  if (p->precision != EXG_PRECISION_F64 && p->precision != EXG_PRECISION_MIXED) return EXG_ERR_INVALID_ARGUMENT;
  if (p->gravity_law == EXG_GRAVITY_PLUMMER && !(p->softening > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  if (!(p->dt > 0.0) || !(p->warp >= 1.0)) return EXG_ERR_INVALID_ARGUMENT;
  for (int32_t i = 0; i < n; ++i)
    if (!bodies[i].kinematic && !(bodies[i].mass > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  for (int32_t k = 0; k < nj; ++k) {
    if (joints[k].law < 0 || joints[k].law > 3) return EXG_ERR_NO_SHADER;
    if (joints[k].a < 0 || joints[k].a >= n || joints[k].b < 0 || joints[k].b >= n || joints[k].a == joints[k].b)
      return EXG_ERR_INVALID_ARGUMENT;
  }
  return EXG_OK;
}

static int upload_bodies(exg_world_s* W, const exg_body_t* bodies, int32_t first, int32_t count) {
  DeviceWorld& w = W->w;
  const int n = w.n;
  std::vector<double> pose(8 * (size_t)count), mom(6 * (size_t)count), mass(count), inertia(9 * (size_t)count),
      size(count);
  std::vector<int> kin(count), diag(count);
  for (int32_t i = 0; i < count; ++i) {
    for (int c = 0; c < 8; ++c) pose[(size_t)c * count + i] = bodies[i].pose[c];
    for (int c = 0; c < 6; ++c) mom[(size_t)c * count + i] = bodies[i].momentum[c];
    for (int c = 0; c < 9; ++c) inertia[(size_t)c * count + i] = bodies[i].inertia[c];
    mass[i] = bodies[i].mass;
    size[i] = bodies[i].size;
    kin[i] = bodies[i].kinematic;
    diag[i] = bodies[i].diagonal;
  }
  cudaStream_t s = W->dev->stream;
  for (int c = 0; c < 8; ++c)
    EXG_CUDA_TRY(cudaMemcpyAsync(w.pose + (size_t)c * n + first, pose.data() + (size_t)c * count, sizeof(double) * count,
                                 cudaMemcpyHostToDevice, s));
  for (int c = 0; c < 6; ++c)
    EXG_CUDA_TRY(cudaMemcpyAsync(w.mom + (size_t)c * n + first, mom.data() + (size_t)c * count, sizeof(double) * count,
                                 cudaMemcpyHostToDevice, s));
  for (int c = 0; c < 9; ++c)
    EXG_CUDA_TRY(cudaMemcpyAsync(w.inertia + (size_t)c * n + first, inertia.data() + (size_t)c * count,
                                 sizeof(double) * count, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.mass + first, mass.data(), sizeof(double) * count, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.size + first, size.data(), sizeof(double) * count, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.kinematic + first, kin.data(), sizeof(int) * count, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.diagonal + first, diag.data(), sizeof(int) * count, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

static int download_bodies(exg_world_s* W, exg_body_t* out, int32_t first, int32_t count) {
  DeviceWorld& w = W->w;
  const int n = w.n;
  std::vector<double> pose(8 * (size_t)count), mom(6 * (size_t)count), mass(count), inertia(9 * (size_t)count),
      size(count);
  std::vector<int> kin(count), diag(count);
  cudaStream_t s = W->dev->stream;
  for (int c = 0; c < 8; ++c)
    EXG_CUDA_TRY(cudaMemcpyAsync(pose.data() + (size_t)c * count, w.pose + (size_t)c * n + first, sizeof(double) * count,
                                 cudaMemcpyDeviceToHost, s));
  for (int c = 0; c < 6; ++c)
    EXG_CUDA_TRY(cudaMemcpyAsync(mom.data() + (size_t)c * count, w.mom + (size_t)c * n + first, sizeof(double) * count,
                                 cudaMemcpyDeviceToHost, s));
  for (int c = 0; c < 9; ++c)
    EXG_CUDA_TRY(cudaMemcpyAsync(inertia.data() + (size_t)c * count, w.inertia + (size_t)c * n + first,
                                 sizeof(double) * count, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(mass.data(), w.mass + first, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(size.data(), w.size + first, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(kin.data(), w.kinematic + first, sizeof(int) * count, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(diag.data(), w.diagonal + first, sizeof(int) * count, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  for (int32_t i = 0; i < count; ++i) {
    for (int c = 0; c < 8; ++c) out[i].pose[c] = pose[(size_t)c * count + i];
    for (int c = 0; c < 6; ++c) out[i].momentum[c] = mom[(size_t)c * count + i];
    for (int c = 0; c < 9; ++c) out[i].inertia[c] = inertia[(size_t)c * count + i];
    out[i].mass = mass[i];
    out[i].size = size[i];
    out[i].kinematic = kin[i];
    out[i].diagonal = diag[i];
  }
  return EXG_OK;
}

template <class T> static int upload_vec(exg_world_s* W, T** dptr, const std::vector<T>& v) {
  int rc = W->alloc(dptr, v.size());
  if (rc != EXG_OK) return rc;
  if (!v.empty())
    EXG_CUDA_TRY(cudaMemcpyAsync(*dptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, W->dev->stream));
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
  W->dev = dev;
  W->p = params[0];
  DeviceWorld& w = W->w;
  const int n = (int)n_total, nj = (int)nj_total;
  w.n = n;
  w.nj = nj;
  w.n_worlds = n_worlds;
  w.precision = params[0].precision;
  w.h_params.assign(params, params + n_worlds);
  std::vector<int> wob(n), woj(nj), law(n_worlds);
  std::vector<double> eps(n_worlds);
  std::vector<exg_joint_t> gj(joints, joints + nj);
  int bo = 0, jo = 0;
  for (int32_t wi = 0; wi < n_worlds; ++wi) {
    w.h_body_off.push_back(bo);
    w.h_n.push_back(body_counts[wi]);
    w.h_joint_off.push_back(jo);
    w.h_nj.push_back(joint_counts[wi]);
    for (int i = 0; i < body_counts[wi]; ++i) wob[bo + i] = wi;
    for (int k = 0; k < joint_counts[wi]; ++k) {
      woj[jo + k] = wi;
      gj[jo + k].a += bo;
      gj[jo + k].b += bo;
    }
    law[wi] = params[wi].gravity_law;
    eps[wi] = params[wi].softening;
    if (params[wi].integrator == EXG_NEWTON) w.any_newton = true; else w.any_explicit = true;
    bo += body_counts[wi];
    jo += joint_counts[wi];
  }
  std::vector<GravItem> items;
  std::vector<int> splits;
  std::vector<long long> poff;
  long long partial_len = 0;
  gravity_plan(w.h_body_off, w.h_n, law, eps, dev->sm_count, items, splits, poff, partial_len);
  w.n_items = (int)items.size();
  int rc = EXG_OK;
#define ALLOC(ptr, cnt) \
  if (rc == EXG_OK) rc = W->alloc(&(ptr), (cnt))
  ALLOC(w.pose, 8 * (size_t)n);
  ALLOC(w.mom, 6 * (size_t)n);
  ALLOC(w.mass, (size_t)n);
  ALLOC(w.inertia, 9 * (size_t)n);
  ALLOC(w.size, (size_t)n);
  ALLOC(w.kinematic, (size_t)n);
  ALLOC(w.diagonal, (size_t)n);
  ALLOC(w.pos_mass, 4 * (size_t)n);
  ALLOC(w.wvel, 6 * (size_t)n);
  ALLOC(w.grav_partial, (size_t)std::max<long long>(partial_len, 1));
  ALLOC(w.conn, 12 * (size_t)nj);
  ALLOC(w.item_head, 1);
#undef ALLOC
  // incidence: per body, its joint ends in joint order (accelerator/mod.rs:289-331)
  std::vector<int> cnt(n + 1, 0), ptr(n + 1, 0), ref(2 * (size_t)nj);
  for (int k = 0; k < nj; ++k) { cnt[gj[k].a]++; cnt[gj[k].b]++; }
  for (int i = 0; i < n; ++i) ptr[i + 1] = ptr[i] + cnt[i];
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int k = 0; k < nj; ++k) { ref[fill[gj[k].a]++] = 2 * k; ref[fill[gj[k].b]++] = 2 * k + 1; }
  if (rc == EXG_OK) rc = upload_vec(W, &w.joints, gj);
  if (rc == EXG_OK) rc = upload_vec(W, &w.world_of_body, wob);
  if (rc == EXG_OK) rc = upload_vec(W, &w.world_of_joint, woj);
  if (rc == EXG_OK) rc = upload_vec(W, &w.inc_ptr, ptr);
  if (rc == EXG_OK) rc = upload_vec(W, &w.inc_ref, ref);
  if (rc == EXG_OK) rc = upload_vec(W, &w.wparams, w.h_params);
  if (rc == EXG_OK) rc = upload_vec(W, &w.w_poff, poff);
  if (rc == EXG_OK) rc = upload_vec(W, &w.w_splits, splits);
  if (rc == EXG_OK) rc = upload_vec(W, &w.w_n, w.h_n);
  if (rc == EXG_OK) rc = upload_vec(W, &w.w_body_off, w.h_body_off);
  if (rc == EXG_OK) rc = upload_vec(W, &w.items, items);
  if (rc == EXG_OK) rc = upload_bodies(W, bodies, 0, n);
  if (rc == EXG_OK && w.any_newton) {
    W->newton = new (std::nothrow) NewtonWorld();
    if (!W->newton) rc = EXG_ERR_OUT_OF_MEMORY;
    else rc = W->newton->init(dev, w, bodies, gj.data(), params[0]);
  }
  if (rc != EXG_OK) { delete W; return rc; }
  *out = W;
  return EXG_OK;
}

int exg_world_create(exg_device_t dev, const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                     const exg_step_params_t* params, exg_world_t* out) {
  return exg_batch_create(dev, 1, &n, &nj, bodies, joints, params, out);
}

int exg_world_destroy(exg_world_t W) {
  if (!W) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  cudaStreamSynchronize(W->dev->stream);
  delete W;
  return EXG_OK;
}

}  // extern "C"

// One step of every world of the batch (Mechanism::step per world, all enqueued asynchronously):
// charges and world twists, gravity, explicit joints and integration, then the implicit islands.
static int enqueue_step(exg_world_s* W, int* kernels) {
  DeviceWorld& w = W->w;
  cudaStream_t s = W->dev->stream;
  uint64_t before = W->dev->launches.load();
  int rc;
  if ((rc = launch_body_pre(W->dev, w, s)) != EXG_OK) return rc;
  if ((rc = launch_gravity_items(W->dev, w.pos_mass, w.size, w.items, w.n_items, w.item_head, w.precision,
                                 w.grav_partial, s)) != EXG_OK)
    return rc;
  if ((rc = launch_joints_plain_world(W->dev, w, s)) != EXG_OK) return rc;
  if ((rc = launch_integrate_explicit(W->dev, w, s)) != EXG_OK) return rc;
  if (W->newton && (rc = W->newton->enqueue(W->dev, w, s)) != EXG_OK) return rc;
  *kernels = (int)(W->dev->launches.load() - before);
  return EXG_OK;
}

static int step_locked(exg_world_s* W, int32_t n_steps) {
  cudaStream_t s = W->dev->stream;
  if (W->dev->profiling) {
    for (int32_t k = 0; k < n_steps; ++k) {
      int kernels = 0;
      int rc = enqueue_step(W, &kernels);
      if (rc != EXG_OK) return rc;
    }
  } else {
    if (!W->graph) {
      // capture one step; replays skip the per-launch host cost
      cudaGraph_t g;
      EXG_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int kernels = 0;
      uint64_t before = W->dev->launches.load();
      int rc = enqueue_step(W, &kernels);
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
    }
  }
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  W->stats.steps += n_steps;
  W->stats.last_spans = 1;
  if (W->newton) {
    int rc = W->newton->read_stats(-1, &W->stats);
    if (rc != EXG_OK) return rc;
    if (W->stats.fatal) return EXG_ERR_FATAL;
  }
  return EXG_OK;
}

extern "C" {

int exg_world_step(exg_world_t W, int32_t n_steps) {
  if (!W || n_steps < 0) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  return step_locked(W, n_steps);
}

int exg_world_get_bodies(exg_world_t W, exg_body_t* out, int32_t n) {
  if (!W || !out || n != W->w.n) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  return download_bodies(W, out, 0, n);
}

int exg_world_set_bodies(exg_world_t W, const exg_body_t* bodies, int32_t n) {
  if (!W || !bodies || n != W->w.n) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  for (int32_t i = 0; i < n; ++i)
    if (!bodies[i].kinematic && !(bodies[i].mass > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  return upload_bodies(W, bodies, 0, n);
}

int exg_batch_get_world(exg_world_t W, int32_t world, exg_body_t* out, int32_t n) {
  if (!W || !out || world < 0 || world >= W->w.n_worlds || n != W->w.h_n[world]) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  return download_bodies(W, out, W->w.h_body_off[world], n);
}

int exg_batch_set_world(exg_world_t W, int32_t world, const exg_body_t* bodies, int32_t n) {
  if (!W || !bodies || world < 0 || world >= W->w.n_worlds || n != W->w.h_n[world]) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  for (int32_t i = 0; i < n; ++i)
    if (!bodies[i].kinematic && !(bodies[i].mass > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  return upload_bodies(W, bodies, W->w.h_body_off[world], n);
}

int exg_world_stats(exg_world_t W, exg_world_stats_t* out) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  *out = W->stats;
  return EXG_OK;
}

int exg_batch_world_stats(exg_world_t W, int32_t world, exg_world_stats_t* out) {
  if (!W || !out || world < 0 || world >= W->w.n_worlds) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  *out = W->stats;
  out->last_spans = 1;
  out->last_newton_iterations = 0;
  out->max_depth_reached = 0;
  out->fatal = 0;
  out->last_residual = 0.0;
  if (W->newton && W->w.h_params[world].integrator == EXG_NEWTON) return W->newton->read_stats(world, out);
  return EXG_OK;
}

int exg_world_phase_cycles(exg_world_t W, int64_t out[8]) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < 8; ++k) out[k] = 0;
  if (!W->newton) return EXG_OK;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  long long tmp[8];
  int rc = W->newton->read_phase_cycles(tmp);
  for (int k = 0; k < 8; ++k) out[k] = tmp[k];
  return rc;
}

int exg_world_energy(exg_world_t W, double* out) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  int n = W->w.n;
  std::vector<exg_body_t> b(n);
  int rc = exg_world_get_bodies(W, b.data(), n);
  if (rc != EXG_OK) return rc;
  std::vector<exg_joint_t> joints(W->w.nj);
  if (W->w.nj > 0) {
    EXG_CUDA_TRY(cudaMemcpy(joints.data(), W->w.joints, sizeof(exg_joint_t) * W->w.nj, cudaMemcpyDeviceToHost));
  }
  double e = 0.0;
  for (int wi = 0; wi < W->w.n_worlds; ++wi) {
    int bo = W->w.h_body_off[wi], jo = W->w.h_joint_off[wi];
    std::vector<exg_joint_t> local(joints.begin() + jo, joints.begin() + jo + W->w.h_nj[wi]);
    for (auto& j : local) { j.a -= bo; j.b -= bo; }
    e += host_world_energy(b.data() + bo, W->w.h_n[wi], local.data(), (int)local.size(), W->w.h_params[wi]);
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
  cudaSetDevice(dev->ordinal);
  int rc = launch_joints_stage(dev, d_joints, nj, d_pose, d_vel, dt, warp, jacobian, d_out, dev->stream);
  if (rc != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(dev->stream));
  return EXG_OK;
}

int exg_gravity_forces(exg_device_t dev, const double* d_pos_mass, const double* d_size, int32_t n, int32_t law, double G,
                       double softening, int32_t precision, double* d_force) {
  if (!dev || n < 0 || (n > 0 && (!d_pos_mass || !d_force))) return EXG_ERR_INVALID_ARGUMENT;
  if (law == EXG_GRAVITY_SIZE_CORE && n > 0 && !d_size) return EXG_ERR_INVALID_ARGUMENT;
  if (law != EXG_GRAVITY_SIZE_CORE && law != EXG_GRAVITY_PLUMMER) return EXG_ERR_INVALID_ARGUMENT;
  if (law == EXG_GRAVITY_PLUMMER && !(softening > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
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
