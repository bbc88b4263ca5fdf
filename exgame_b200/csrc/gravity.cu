// All-pairs gravity (crates/newton/src/gravity.rs:110-140, 438-450 and the Plummer law of the
// synthetic workloads).
//
// Layout and decomposition:
//   * bodies arrive as double4 (x, y, z, m); kinematic bodies carry m = 0 and so exert and
//     feel no force (the reference gives them no gravitational charge, gravity.rs:485-497);
//   * a CTA owns an i-tile of TILE bodies (one body per thread) and one of `splits` j-ranges;
//     j-tiles of TILE bodies are staged in shared memory and read back as broadcasts;
//   * the CTA writes its partial sum  sum_j m_j r_ij / core^3  to partial[split][3][n]; the
//     consumer adds the splits in index order and multiplies by G m_i, so the result does not
//     depend on scheduling (no atomics).
// Precision: R = double is the plain path. R = float is the mixed path: positions are taken
// relative to the i-tile's first body (one double subtraction per staged j-body, amortised over
// the tile), pair terms are FP32 with the hardware reciprocal square root, and each j-tile's
// FP32 partial is flushed into an FP64 accumulator, so rounding does not grow with n.
#include "exg_internal.cuh"

namespace {

template <class R> __device__ __forceinline__ R rsqrt_r(R x);
template <> __device__ __forceinline__ double rsqrt_r<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float rsqrt_r<float>(float x) { return rsqrtf(x); }

template <class R> struct Vec4;
template <> struct Vec4<double> { typedef double4 T; };
template <> struct Vec4<float> { typedef float4 T; };

// LAW 1 = size core (reference), 2 = Plummer
template <class R, int LAW, int TILE>
__global__ void __launch_bounds__(TILE) k_gravity(const double4* __restrict__ pm, const double* __restrict__ size, int n,
                                                  R eps2, int split_len, double* __restrict__ partial) {
  typedef typename Vec4<R>::T V4;
  __shared__ V4 tile[TILE];
  __shared__ R tsz2[LAW == 1 ? TILE : 1];
  __shared__ R tisz3[LAW == 1 ? TILE : 1];
  const int i = blockIdx.x * TILE + threadIdx.x;
  const int split = blockIdx.y;
  const int j0 = split * split_len;
  const int j1 = min(n, j0 + split_len);
  // reference point: first body of the i-tile (mixed path only)
  double4 c = make_double4(0.0, 0.0, 0.0, 0.0);
  if (sizeof(R) == 4) c = pm[blockIdx.x * TILE];
  double4 pi = (i < n) ? pm[i] : make_double4(0.0, 0.0, 0.0, 0.0);
  const R xi = R(pi.x - c.x), yi = R(pi.y - c.y), zi = R(pi.z - c.z);
  R sz2_i = R(0), isz3_i = R(0);
  if (LAW == 1 && i < n) {
    double s = size[i];
    sz2_i = R(s * s);
    isz3_i = R(1.0 / (s * s * s));
  }
  double dax = 0.0, day = 0.0, daz = 0.0;
  for (int base = j0; base < j1; base += TILE) {
    const int j = base + threadIdx.x;
    if (j < j1) {
      double4 q = pm[j];
      V4 t;
      t.x = R(q.x - c.x); t.y = R(q.y - c.y); t.z = R(q.z - c.z); t.w = R(q.w);
      tile[threadIdx.x] = t;
      if (LAW == 1) {
        double s = size[j];
        tsz2[threadIdx.x] = R(s * s);
        tisz3[threadIdx.x] = R(1.0 / (s * s * s));
      }
    } else {
      V4 t; t.x = R(0); t.y = R(0); t.z = R(0); t.w = R(0);
      tile[threadIdx.x] = t;
      if (LAW == 1) { tsz2[threadIdx.x] = R(1); tisz3[threadIdx.x] = R(0); }
    }
    __syncthreads();
    R ax = R(0), ay = R(0), az = R(0);
    if (LAW == 2) {
#pragma unroll 8
      for (int k = 0; k < TILE; ++k) {
        V4 q = tile[k];
        R dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
        R s2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
        R inv = rsqrt_r<R>(s2);
        R s = q.w * (inv * inv * inv);
        ax = fma(dx, s, ax); ay = fma(dy, s, ay); az = fma(dz, s, az);
      }
    } else {
      const int jb = base;
#pragma unroll 4
      for (int k = 0; k < TILE; ++k) {
        V4 q = tile[k];
        R dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
        R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
        // core radius of the higher-slot body (gravity.rs:126-131)
        bool j_hi = (jb + k) > i;
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
  if (i < n) {
    double* p = partial + (size_t)split * 3 * n;
    p[i] = dax; p[n + i] = day; p[2 * n + i] = daz;
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

template <class R, int LAW>
int launch_t(exg_device_s* dev, const double* pos_mass, const double* size, int n, double softening, GravityShape sh,
             double* partial, cudaStream_t s) {
  int split_len = (n + sh.splits - 1) / sh.splits;
  split_len = ((split_len + sh.tile - 1) / sh.tile) * sh.tile;
  int splits = (n + split_len - 1) / split_len;
  dim3 grid((n + sh.tile - 1) / sh.tile, splits);
  R eps2 = R(softening * softening);
  const double4* pm = reinterpret_cast<const double4*>(pos_mass);
  int _tok = prof_begin(dev, PROF_GRAVITY, s);
  switch (sh.tile) {
    case 64: k_gravity<R, LAW, 64><<<grid, 64, 0, s>>>(pm, size, n, eps2, split_len, partial); break;
    case 128: k_gravity<R, LAW, 128><<<grid, 128, 0, s>>>(pm, size, n, eps2, split_len, partial); break;
    default: k_gravity<R, LAW, 256><<<grid, 256, 0, s>>>(pm, size, n, eps2, split_len, partial); break;
  }
  prof_end(dev, _tok, s);
  if (splits < sh.splits) {
    // the unused split slots must read as zero
    cudaMemsetAsync(partial + (size_t)splits * 3 * n, 0, sizeof(double) * 3 * (size_t)n * (sh.splits - splits), s);
  }
  return exg_after_launch(dev);
}

}  // namespace

GravityShape gravity_pick_shape(int n, int sm_count, int precision) {
  GravityShape sh;
  int sms = sm_count > 0 ? sm_count : 148;
  if (n >= sms * 256 * 2) sh.tile = 256;
  else if (n >= sms * 128) sh.tile = 128;
  else sh.tile = 64;
  int itiles = (n + sh.tile - 1) / sh.tile;
  int target = sms * 8;
  int splits = (target + itiles - 1) / itiles;
  int max_splits = (n + sh.tile - 1) / sh.tile;
  if (splits > max_splits) splits = max_splits;
  if (splits > 32) splits = 32;
  if (splits < 1) splits = 1;
  sh.splits = splits;
  (void)precision;
  return sh;
}

int launch_gravity(exg_device_s* dev, const double* pos_mass, const double* size, int n, int law, double softening,
                   int precision, GravityShape shape, double* partial, cudaStream_t s) {
  if (n <= 0) return EXG_OK;
  if (law == EXG_GRAVITY_PLUMMER && !(softening > 0.0)) return EXG_ERR_INVALID_ARGUMENT;
  if (precision == EXG_PRECISION_MIXED) {
    if (law == EXG_GRAVITY_PLUMMER) return launch_t<float, 2>(dev, pos_mass, size, n, softening, shape, partial, s);
    return launch_t<float, 1>(dev, pos_mass, size, n, softening, shape, partial, s);
  }
  if (law == EXG_GRAVITY_PLUMMER) return launch_t<double, 2>(dev, pos_mass, size, n, softening, shape, partial, s);
  return launch_t<double, 1>(dev, pos_mass, size, n, softening, shape, partial, s);
}

int launch_gravity_reduce(exg_device_s* dev, const double* partial, const double* pos_mass, int n, int splits, double G,
                          double* force_out, cudaStream_t s) {
  if (n <= 0) return EXG_OK;
  k_gravity_reduce<<<(n + 255) / 256, 256, 0, s>>>(partial, reinterpret_cast<const double4*>(pos_mass), n, splits, G,
                                                   force_out);
  return exg_after_launch(dev);
}
