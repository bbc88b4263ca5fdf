// All-pairs gravity over a batch of worlds (crates/newton/src/gravity.rs:110-140, 438-450, and
// the Plummer law of the synthetic workloads).
//
// Work decomposition: a work item is an i-tile of kGravTile bodies of one world against a
// j-range of the same world (bodies of different worlds never interact). Items are listed
// largest-first and pulled by persistent CTAs through an atomic counter, so worlds of very
// uneven size (8 .. 8192 bodies) share the GPU without a tail of idle SMs. Within an item each
// thread owns one i-body; j-bodies are staged through shared memory in tiles of kGravTile and
// read back as broadcasts. The item writes its partial sum  sum_j m_j r_ij / core^3  to its own
// slot; consumers add a world's splits in index order and multiply by G m_i, so results do not
// depend on scheduling (no atomics on the data).
//
// Kinematic bodies carry m = 0 in the charge array and so exert no force (the reference gives
// them no gravitational charge, gravity.rs:485-497).
//
// Precision: R = double is the plain path. R = float is the mixed path: positions are taken
// relative to the item's first i-body (one double subtraction per staged j-body, amortised over
// the tile), pair terms are FP32 with the hardware reciprocal square root, and each j-tile's FP32
// partial is flushed into an FP64 accumulator, so rounding does not grow with the world size.
#include <algorithm>
#include <mutex>
#include "exg_internal.cuh"

namespace {

template <class R> __device__ __forceinline__ R rsqrt_r(R x);
template <> __device__ __forceinline__ double rsqrt_r<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float rsqrt_r<float>(float x) { return rsqrtf(x); }

template <class R> struct Vec4;
template <> struct Vec4<double> { typedef double4 T; };
template <> struct Vec4<float> { typedef float4 T; };

template <class R>
__global__ void __launch_bounds__(kGravTile) k_gravity_items(const double4* __restrict__ pm, const double* __restrict__ size,
                                                             const GravItem* __restrict__ items, int n_items,
                                                             int* __restrict__ head, double* __restrict__ partial) {
  constexpr int T = kGravTile;
  typedef typename Vec4<R>::T V4;
  __shared__ V4 tile[T];
  __shared__ R tsz2[T];
  __shared__ R tisz3[T];
  __shared__ int cur;
  for (;;) {
    if (threadIdx.x == 0) cur = atomicAdd(head, 1);
    __syncthreads();
    const int it = cur;
    __syncthreads();
    if (it >= n_items) return;
    const GravItem g = items[it];
    const int il = g.i0 + threadIdx.x;
    const bool valid = il < g.n;
    const double4* wpm = pm + g.body_off;
    double4 c = make_double4(0.0, 0.0, 0.0, 0.0);
    if (sizeof(R) == 4) c = wpm[g.i0];
    const double4 pi = valid ? wpm[il] : c;
    const R xi = R(pi.x - c.x), yi = R(pi.y - c.y), zi = R(pi.z - c.z);
    const bool core_law = g.law == EXG_GRAVITY_SIZE_CORE;
    R sz2_i = R(0), isz3_i = R(0);
    if (core_law && valid) {
      double s = size[g.body_off + il];
      sz2_i = R(s * s);
      isz3_i = R(1.0 / (s * s * s));
    }
    const R eps2 = R(g.eps2);
    double dax = 0.0, day = 0.0, daz = 0.0;
    for (int base = g.j0; base < g.j1; base += T) {
      const int j = base + threadIdx.x;
      V4 t;
      if (j < g.j1) {
        double4 q = wpm[j];
        t.x = R(q.x - c.x); t.y = R(q.y - c.y); t.z = R(q.z - c.z); t.w = R(q.w);
        if (core_law) {
          double s = size[g.body_off + j];
          tsz2[threadIdx.x] = R(s * s);
          tisz3[threadIdx.x] = R(1.0 / (s * s * s));
        }
      } else {
        t.x = R(0); t.y = R(0); t.z = R(0); t.w = R(0);
        if (core_law) { tsz2[threadIdx.x] = R(1); tisz3[threadIdx.x] = R(0); }
      }
      tile[threadIdx.x] = t;
      __syncthreads();
      R ax = R(0), ay = R(0), az = R(0);
      if (!core_law) {
#pragma unroll 8
        for (int k = 0; k < T; ++k) {
          V4 q = tile[k];
          R dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
          R s2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
          R inv = rsqrt_r<R>(s2);
          R s = q.w * (inv * inv * inv);
          ax = fma(dx, s, ax); ay = fma(dy, s, ay); az = fma(dz, s, az);
        }
      } else {
#pragma unroll 4
        for (int k = 0; k < T; ++k) {
          V4 q = tile[k];
          R dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
          R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
          // core radius of the higher-slot body (gravity.rs:126-131)
          bool j_hi = (base + k) > il;
          R sz2 = j_hi ? tsz2[k] : sz2_i;
          R isz3 = j_hi ? tisz3[k] : isz3_i;
          R inv = rsqrt_r<R>(r2);
          R sd = (r2 >= sz2) ? inv * inv * inv : isz3;
          // coincident bodies exert nothing (|d| < 1e-9, gravity.rs:119-122)
          R s = (r2 < R(1e-18)) ? R(0) : q.w * sd;
          ax = fma(dx, s, ax); ay = fma(dy, s, ay); az = fma(dz, s, az);
        }
      }
      dax += double(ax); day += double(ay); daz += double(az);
      __syncthreads();
    }
    if (valid) {
      double* p = partial + g.out_off;
      p[il] = dax; p[g.n + il] = day; p[2 * (size_t)g.n + il] = daz;
    }
  }
}

__global__ void k_gravity_reduce(const double* __restrict__ partial, const double4* __restrict__ pm, int n, int splits,
                                 double G, double* __restrict__ force) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double gm = G * pm[i].w;
  for (int c = 0; c < 3; ++c) {
    double acc = 0.0;
    for (int s = 0; s < splits; ++s) acc += partial[(size_t)s * 3 * n + (size_t)c * n + i];
    force[3 * i + c] = gm * acc;
  }
}

}  // namespace

void gravity_plan(const std::vector<int>& body_off, const std::vector<int>& n, const std::vector<int>& law,
                  const std::vector<double>& eps, int sm_count, std::vector<GravItem>& items, std::vector<int>& splits,
                  std::vector<long long>& poff, long long& partial_len) {
  // The j-range of an item depends on the world's own size only (the smallest power of two
  // >= n/8, clamped to [128, 2048]), so a world's arithmetic — and its result, bit for bit — is
  // the same stepped alone or inside any batch.
  const int T = kGravTile;
  const int W = (int)n.size();
  (void)sm_count;
  splits.assign(W, 0);
  poff.assign(W, 0);
  items.clear();
  long long run = 0;
  std::vector<std::pair<double, GravItem>> tmp;
  for (int w = 0; w < W; ++w) {
    if (law[w] == EXG_GRAVITY_OFF || n[w] <= 1) continue;
    const int nw = n[w];
    int L = T;
    while (L < 2048 && L * 8 < nw) L *= 2;
    const int itiles = (nw + T - 1) / T;
    const int sp = (nw + L - 1) / L;
    splits[w] = sp;
    poff[w] = run;
    for (int s = 0; s < sp; ++s)
      for (int t = 0; t < itiles; ++t) {
        GravItem g;
        g.body_off = body_off[w];
        g.n = nw;
        g.i0 = t * T;
        g.j0 = s * L;
        g.j1 = std::min(nw, g.j0 + L);
        g.law = law[w];
        g.eps2 = eps[w] * eps[w];
        g.out_off = run + (long long)s * 3 * nw;
        double work = double(std::min(T, nw - g.i0)) * (g.j1 - g.j0);
        tmp.push_back({work, g});
      }
    run += (long long)sp * 3 * nw;
  }
  std::stable_sort(tmp.begin(), tmp.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  for (auto& x : tmp) items.push_back(x.second);
  partial_len = run;
}

int launch_gravity_items(exg_device_s* dev, const double* pos_mass, const double* size, const GravItem* items, int n_items,
                         int* head, int precision, double* partial, cudaStream_t s) {
  if (n_items <= 0) return EXG_OK;
  EXG_CUDA_TRY(cudaMemsetAsync(head, 0, sizeof(int), s));
  int sms = dev->sm_count > 0 ? dev->sm_count : 148;
  int grid = std::min(n_items, sms * 12);
  const double4* pm = reinterpret_cast<const double4*>(pos_mass);
  int tok = prof_begin(dev, PROF_GRAVITY, s);
  if (precision == EXG_PRECISION_MIXED)
    k_gravity_items<float><<<grid, kGravTile, 0, s>>>(pm, size, items, n_items, head, partial);
  else
    k_gravity_items<double><<<grid, kGravTile, 0, s>>>(pm, size, items, n_items, head, partial);
  prof_end(dev, tok, s);
  return exg_after_launch(dev);
}

int launch_gravity_reduce(exg_device_s* dev, const double* partial, const double* pos_mass, int n, int splits, double G,
                          double* force_out, cudaStream_t s) {
  if (n <= 0) return EXG_OK;
  k_gravity_reduce<<<(n + 255) / 256, 256, 0, s>>>(partial, reinterpret_cast<const double4*>(pos_mass), n, splits, G,
                                                   force_out);
  return exg_after_launch(dev);
}

// ── the no-allocation variant of the gravity stage ─────────────────────────────
// Its scratch is a file-scope device array sized for EXG_NOALLOC_MAX_BODIES bodies: the work
// items, the per-split partial sums and the scheduler counter. The host side never names the
// array as a device address: it asks the runtime for the address once per device and passes
// that to the kernels.
namespace {
constexpr int kNoAllocMaxItems = ((EXG_NOALLOC_MAX_BODIES + kGravTile - 1) / kGravTile) * 8;  // splits <= 8 here
constexpr size_t kNoAllocPartialDoubles = (size_t)8 * 3 * EXG_NOALLOC_MAX_BODIES;
constexpr size_t kNoAllocHeadBytes = 256;
constexpr size_t kNoAllocItemBytes = ((sizeof(GravItem) * kNoAllocMaxItems + 255) / 256) * 256;
constexpr size_t kNoAllocBytes = kNoAllocHeadBytes + kNoAllocItemBytes + kNoAllocPartialDoubles * sizeof(double);
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {nullptr};  // device address of the scratch array, per device ordinal

// Resolve the scratch array's device address on `ordinal` (that device must be current).
int noalloc_scratch(int ordinal, unsigned char** out) {
  if (ordinal < 0 || ordinal >= 256) return EXG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[ordinal]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      exg_internal_set_cuda_error(e, "cudaGetSymbolAddress(no-allocation gravity scratch)");
      return EXG_ERR_BACKEND;
    }
    g_noalloc_addr[ordinal] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[ordinal]);
  return EXG_OK;
}
}  // namespace

extern "C" int exg_gravity_forces_noalloc(exg_device_t dev, const double* d_pos_mass, const double* d_size, int32_t n,
                                          int32_t law, double G, double softening, int32_t precision, double* d_force) {
  if (!dev || n < 0 || (n > 0 && (!d_pos_mass || !d_force))) return EXG_ERR_INVALID_ARGUMENT;
  if (n > EXG_NOALLOC_MAX_BODIES) return EXG_ERR_INVALID_ARGUMENT;
  if (law == EXG_GRAVITY_SIZE_CORE && n > 0 && !d_size) return EXG_ERR_INVALID_ARGUMENT;
  if (law != EXG_GRAVITY_SIZE_CORE && law != EXG_GRAVITY_PLUMMER) return EXG_ERR_INVALID_ARGUMENT;
  if (law == EXG_GRAVITY_PLUMMER && !(softening > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  if (n == 0) return EXG_OK;
  std::lock_guard<std::mutex> lock(dev->mu);
  EXG_CUDA_TRY(cudaSetDevice(dev->ordinal));
  cudaStream_t s = dev->stream;
  if (n == 1) {
    EXG_CUDA_TRY(cudaMemsetAsync(d_force, 0, 3 * sizeof(double), s));
    EXG_CUDA_TRY(cudaStreamSynchronize(s));
    return EXG_OK;
  }
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(dev->ordinal, &base);
  if (rc != EXG_OK) return rc;
  std::vector<GravItem> items;
  std::vector<int> splits;
  std::vector<long long> poff;
  long long plen = 0;
  gravity_plan({0}, {n}, {law}, {softening}, dev->sm_count, items, splits, poff, plen);
  if ((long long)items.size() > kNoAllocMaxItems || plen > (long long)kNoAllocPartialDoubles)
    return EXG_ERR_INVALID_ARGUMENT;
  int* head = reinterpret_cast<int*>(base);
  GravItem* d_items = reinterpret_cast<GravItem*>(base + kNoAllocHeadBytes);
  double* partial = reinterpret_cast<double*>(base + kNoAllocHeadBytes + kNoAllocItemBytes);
  EXG_CUDA_TRY(cudaMemcpyAsync(d_items, items.data(), sizeof(GravItem) * items.size(), cudaMemcpyHostToDevice, s));
  rc = launch_gravity_items(dev, d_pos_mass, d_size, d_items, (int)items.size(), head, precision, partial, s);
  if (rc == EXG_OK) rc = launch_gravity_reduce(dev, partial, d_pos_mass, n, splits[0], G, d_force, s);
  // the host item table must outlive the copy, so wait here in every case
  cudaError_t e = cudaStreamSynchronize(s);
  if (rc != EXG_OK) return rc;
  if (e != cudaSuccess) {
    exg_internal_set_cuda_error(e, "no-allocation gravity");
    return EXG_ERR_BACKEND;
  }
  return EXG_OK;
}
