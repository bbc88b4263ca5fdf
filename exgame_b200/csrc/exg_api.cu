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

static int validate_world(const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                          const exg_step_params_t* p) {
  if (n < 0 || nj < 0 || (n > 0 && !bodies) || (nj > 0 && !joints) || !p) return EXG_ERR_INVALID_ARGUMENT;
  if (p->integrator < 0 || p->integrator > EXG_NEWTON) return EXG_ERR_INVALID_ARGUMENT;
  if (p->gravity_law < 0 || p->gravity_law > EXG_GRAVITY_PLUMMER) return EXG_ERR_INVALID_ARGUMENT;
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

static int upload_bodies(exg_world_s* W, const exg_body_t* bodies, int32_t n) {
  std::vector<double> pose(8 * (size_t)n), mom(6 * (size_t)n), mass(n), inertia(9 * (size_t)n), size(n);
  std::vector<int> kin(n), diag(n);
  for (int32_t i = 0; i < n; ++i) {
    for (int c = 0; c < 8; ++c) pose[(size_t)c * n + i] = bodies[i].pose[c];
    for (int c = 0; c < 6; ++c) mom[(size_t)c * n + i] = bodies[i].momentum[c];
    for (int c = 0; c < 9; ++c) inertia[(size_t)c * n + i] = bodies[i].inertia[c];
    mass[i] = bodies[i].mass;
    size[i] = bodies[i].size;
    kin[i] = bodies[i].kinematic;
    diag[i] = bodies[i].diagonal;
  }
  cudaStream_t s = W->dev->stream;
  DeviceWorld& w = W->w;
  EXG_CUDA_TRY(cudaMemcpyAsync(w.pose, pose.data(), sizeof(double) * pose.size(), cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.mom, mom.data(), sizeof(double) * mom.size(), cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.mass, mass.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.inertia, inertia.data(), sizeof(double) * inertia.size(), cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.size, size.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.kinematic, kin.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(w.diagonal, diag.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  return EXG_OK;
}

int exg_world_create(exg_device_t dev, const exg_body_t* bodies, int32_t n, const exg_joint_t* joints, int32_t nj,
                     const exg_step_params_t* params, exg_world_t* out) {
  if (!dev || !out) return EXG_ERR_INVALID_ARGUMENT;
  int st = validate_world(bodies, n, joints, nj, params);
  if (st != EXG_OK) return st;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
  exg_world_s* W = new (std::nothrow) exg_world_s();
  if (!W) return EXG_ERR_OUT_OF_MEMORY;
  W->dev = dev;
  W->p = *params;
  DeviceWorld& w = W->w;
  w.n = n;
  w.nj = nj;
  w.gshape = gravity_pick_shape(n, dev->sm_count, params->precision);
  w.grav_splits = w.gshape.splits;
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
  ALLOC(w.joints, (size_t)nj);
  ALLOC(w.inc_ptr, (size_t)n + 1);
  ALLOC(w.inc_ref, 2 * (size_t)nj);
  ALLOC(w.pos_mass, 4 * (size_t)n);
  ALLOC(w.wvel, 6 * (size_t)n);
  ALLOC(w.grav_partial, (size_t)w.grav_splits * 3 * n);
  ALLOC(w.conn, 12 * (size_t)nj);
#undef ALLOC
  if (rc != EXG_OK) { delete W; return rc; }
  // incidence: per body, its joint ends in joint order (accelerator/mod.rs:289-331)
  std::vector<int> cnt(n + 1, 0), ptr(n + 1, 0), ref(2 * (size_t)nj);
  for (int32_t k = 0; k < nj; ++k) { cnt[joints[k].a]++; cnt[joints[k].b]++; }
  for (int32_t i = 0; i < n; ++i) ptr[i + 1] = ptr[i] + cnt[i];
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int32_t k = 0; k < nj; ++k) { ref[fill[joints[k].a]++] = 2 * k; ref[fill[joints[k].b]++] = 2 * k + 1; }
  cudaStream_t s = dev->stream;
  if (nj > 0) {
    if (cudaMemcpyAsync(w.joints, joints, sizeof(exg_joint_t) * nj, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(w.inc_ref, ref.data(), sizeof(int) * ref.size(), cudaMemcpyHostToDevice, s) != cudaSuccess)
      rc = EXG_ERR_BACKEND;
  }
  if (rc == EXG_OK && cudaMemcpyAsync(w.inc_ptr, ptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s) != cudaSuccess)
    rc = EXG_ERR_BACKEND;
  if (rc == EXG_OK) rc = upload_bodies(W, bodies, n);
  if (rc == EXG_OK && params->integrator == EXG_NEWTON) {
    W->newton = new (std::nothrow) NewtonWorld();
    if (!W->newton) rc = EXG_ERR_OUT_OF_MEMORY;
    else rc = W->newton->init(dev, w, bodies, joints, *params);
  }
  if (rc != EXG_OK) { delete W; return rc; }
  *out = W;
  return EXG_OK;
}

int exg_world_destroy(exg_world_t W) {
  if (!W) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  cudaStreamSynchronize(W->dev->stream);
  delete W;
  return EXG_OK;
}

// One explicit step's launches (bridge.rs:19-63 over Mechanism::step).
static int enqueue_explicit_step(exg_world_s* W, int* kernels) {
  DeviceWorld& w = W->w;
  const exg_step_params_t& p = W->p;
  cudaStream_t s = W->dev->stream;
  int k = 0, rc;
  if ((rc = launch_body_pre(W->dev, w, s)) != EXG_OK) return rc;
  ++k;
  bool grav = p.gravity_law != EXG_GRAVITY_OFF && w.n > 1;
  if (grav) {
    if ((rc = launch_gravity(W->dev, w.pos_mass, w.size, w.n, p.gravity_law, p.softening, p.precision, w.gshape,
                             w.grav_partial, s)) != EXG_OK)
      return rc;
    ++k;
  }
  if (w.nj > 0) {
    if ((rc = launch_joints_plain_world(W->dev, w, p.dt, p.warp, s)) != EXG_OK) return rc;
    ++k;
  }
  if ((rc = launch_integrate_explicit(W->dev, w, p.integrator, grav ? 1 : 0, p.G, p.dt, s)) != EXG_OK) return rc;
  ++k;
  *kernels = k;
  return EXG_OK;
}

int exg_world_step(exg_world_t W, int32_t n_steps) {
  if (!W || n_steps < 0) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  if (W->p.integrator == EXG_NEWTON) {
    int rc = W->newton->step(W->dev, W->w, W->p, n_steps, &W->stats);
    if (rc == EXG_OK) W->stats.steps += n_steps;
    return rc;
  }
  cudaStream_t s = W->dev->stream;
  if (W->dev->profiling) {
    // direct launches so each kernel can be bracketed by events
    for (int32_t k = 0; k < n_steps; ++k) {
      int kernels = 0;
      int rc = enqueue_explicit_step(W, &kernels);
      if (rc != EXG_OK) return rc;
    }
    EXG_CUDA_TRY(cudaStreamSynchronize(s));
    W->stats.steps += n_steps;
    W->stats.last_spans = 1;
    return EXG_OK;
  }
  if (!W->graph) {
    // capture one step; replays skip the per-launch host cost
    cudaGraph_t g;
    EXG_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int kernels = 0;
    uint64_t before = W->dev->launches.load();
    int rc = enqueue_explicit_step(W, &kernels);
    W->dev->launches.store(before);  // captured, not yet launched
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc != EXG_OK) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
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
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  W->stats.steps += n_steps;
  W->stats.last_spans = 1;
  return EXG_OK;
}

int exg_world_get_bodies(exg_world_t W, exg_body_t* out, int32_t n) {
  if (!W || !out || n != W->w.n) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  DeviceWorld& w = W->w;
  std::vector<double> pose(8 * (size_t)n), mom(6 * (size_t)n), mass(n), inertia(9 * (size_t)n), size(n);
  std::vector<int> kin(n), diag(n);
  cudaStream_t s = W->dev->stream;
  EXG_CUDA_TRY(cudaMemcpyAsync(pose.data(), w.pose, sizeof(double) * pose.size(), cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(mom.data(), w.mom, sizeof(double) * mom.size(), cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(mass.data(), w.mass, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(inertia.data(), w.inertia, sizeof(double) * inertia.size(), cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(size.data(), w.size, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(kin.data(), w.kinematic, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaMemcpyAsync(diag.data(), w.diagonal, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  EXG_CUDA_TRY(cudaStreamSynchronize(s));
  for (int32_t i = 0; i < n; ++i) {
    for (int c = 0; c < 8; ++c) out[i].pose[c] = pose[(size_t)c * n + i];
    for (int c = 0; c < 6; ++c) out[i].momentum[c] = mom[(size_t)c * n + i];
    for (int c = 0; c < 9; ++c) out[i].inertia[c] = inertia[(size_t)c * n + i];
    out[i].mass = mass[i];
    out[i].size = size[i];
    out[i].kinematic = kin[i];
    out[i].diagonal = diag[i];
  }
  return EXG_OK;
}

int exg_world_set_bodies(exg_world_t W, const exg_body_t* bodies, int32_t n) {
  if (!W || !bodies || n != W->w.n) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(W->dev->mu);
  cudaSetDevice(W->dev->ordinal);
  for (int32_t i = 0; i < n; ++i)
    if (!bodies[i].kinematic && !(bodies[i].mass > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  return upload_bodies(W, bodies, n);
}

int exg_world_stats(exg_world_t W, exg_world_stats_t* out) {
  if (!W || !out) return EXG_ERR_INVALID_ARGUMENT;
  *out = W->stats;
  return EXG_OK;
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
  *out = host_world_energy(b.data(), n, joints.data(), W->w.nj, W->p);
  return EXG_OK;
}

int exg_motor_exp(const double twist[6], double dt, double out[8]) {
  if (!twist || !out) return EXG_ERR_INVALID_ARGUMENT;
  double b[6];
  exg::screw_from6(twist, b);
  exg::twist_exp(b, dt, out);
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
  if (n == 0) return EXG_OK;
  std::lock_guard<std::mutex> lock(dev->mu);
  cudaSetDevice(dev->ordinal);
  GravityShape sh = gravity_pick_shape(n, dev->sm_count, precision);
  double* partial = nullptr;
  EXG_CUDA_TRY(cudaMallocAsync(&partial, sizeof(double) * 3 * (size_t)n * sh.splits, dev->stream));
  int rc = launch_gravity(dev, d_pos_mass, d_size, n, law, softening, precision, sh, partial, dev->stream);
  if (rc == EXG_OK) rc = launch_gravity_reduce(dev, partial, d_pos_mass, n, sh.splits, G, d_force, dev->stream);
  cudaFreeAsync(partial, dev->stream);
  if (rc != EXG_OK) return rc;
  EXG_CUDA_TRY(cudaStreamSynchronize(dev->stream));
  return EXG_OK;
}

}  // extern "C"
