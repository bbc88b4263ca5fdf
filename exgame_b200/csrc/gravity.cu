// All-pairs gravity over a batch of worlds (crates/newton/src/gravity.rs:110-140, 438-450, and
// the Plummer law of the synthetic workloads).
//
// Work decomposition: a work item is an i-tile of kGravTile bodies of one world against a
// j-range of the same world (bodies of different worlds never interact). Items are listed
// largest-first and pulled by persistent CTAs through an atomic counter, so worlds of very
// uneven size (8 .. 8192 bodies) share the GPU without a tail of idle SMs. j-bodies are staged
// through shared memory in tiles of kGravTile and read back as broadcasts. The item writes its
// partial sum  sum_j m_j r_ij / core^3  to its own slot; consumers add a world's splits in index
// order and multiply by G m_i, so results do not depend on scheduling (no atomics on the data).
//
// Kinematic bodies carry m = 0 in the charge array and so exert no force (the reference gives
// them no gravitational charge, gravity.rs:485-497).
//
// Precision: k_gravity_items<double> is the plain (F64) path, two i-bodies per thread.
// k_gravity_items_mixed is the mixed path (one warp per item, four i-bodies per thread as two
// FP32x2 packs): positions relative to the item's first i-body (one double subtraction per staged
// body), FP32 pair terms with the hardware reciprocal square root, each j-tile's FP32 partial
// flushed into an FP64 accumulator so rounding does not grow with the world size; its COMP form
// (precision MIXED) also carries the FP32 remainder of every relative position.
#include <algorithm>
#include <mutex>
#include "exg_internal.cuh"

namespace {

template <class R> __device__ __forceinline__ R rsqrt_r(R x);
template <> __device__ __forceinline__ double rsqrt_r<double>(double x) { return rsqrt(x); }

template <class R> struct Vec4;
template <> struct Vec4<double> { typedef double4 T; };
template <> struct Vec4<float> { typedef float4 T; };

// One CTA of kGravThreads threads owns an i-tile of kGravTile = 2 * kGravThreads bodies (thread t:
// bodies i0 + t and i0 + t + kGravThreads), so each shared-memory broadcast of a j-body feeds two
// pair evaluations. Every i-body still sums its j-range tile by tile in j order, then flushes the
// tile's FP32 partial into FP64.
constexpr int kGravThreads = kGravTile / 2;

template <class R>
__global__ void __launch_bounds__(kGravThreads) k_gravity_items(const double4* __restrict__ pm,
                                                                const double* __restrict__ size,
                                                                const GravItem* __restrict__ items, int n_items,
                                                                int* __restrict__ head, double* __restrict__ partial,
                                                                const int* __restrict__ world_of_body,
                                                                const int* __restrict__ w_active) {
  constexpr int T = kGravTile;
  constexpr int H = kGravThreads;
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
    if (w_active && !w_active[world_of_body[g.body_off]]) continue;  // the world holds this step
    const int il0 = g.i0 + threadIdx.x, il1 = il0 + H;
    const bool v0 = il0 < g.n, v1 = il1 < g.n;
    const double4* wpm = pm + g.body_off;
    double4 c = make_double4(0.0, 0.0, 0.0, 0.0);
    if (sizeof(R) == 4) c = wpm[g.i0];
    const double4 p0 = v0 ? wpm[il0] : c, p1 = v1 ? wpm[il1] : c;
    const R x0 = R(p0.x - c.x), y0 = R(p0.y - c.y), z0 = R(p0.z - c.z);
    const R x1 = R(p1.x - c.x), y1 = R(p1.y - c.y), z1 = R(p1.z - c.z);
    const bool core_law = g.law == EXG_GRAVITY_SIZE_CORE;
    R sz2_0 = R(0), isz3_0 = R(0), sz2_1 = R(0), isz3_1 = R(0);
    if (core_law) {
      if (v0) { double s = size[g.body_off + il0]; sz2_0 = R(s * s); isz3_0 = R(1.0 / (s * s * s)); }
      if (v1) { double s = size[g.body_off + il1]; sz2_1 = R(s * s); isz3_1 = R(1.0 / (s * s * s)); }
    }
    const R eps2 = R(g.eps2);
    double da0x = 0.0, da0y = 0.0, da0z = 0.0, da1x = 0.0, da1y = 0.0, da1z = 0.0;
    for (int base = g.j0; base < g.j1; base += T) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int slot = threadIdx.x + h * H;
        const int j = base + slot;
        V4 t;
        if (j < g.j1) {
          double4 q = wpm[j];
          t.x = R(q.x - c.x); t.y = R(q.y - c.y); t.z = R(q.z - c.z); t.w = R(q.w);
          if (core_law) {
            double s = size[g.body_off + j];
            tsz2[slot] = R(s * s);
            tisz3[slot] = R(1.0 / (s * s * s));
          }
        } else {
          t.x = R(0); t.y = R(0); t.z = R(0); t.w = R(0);
          if (core_law) { tsz2[slot] = R(1); tisz3[slot] = R(0); }
        }
        tile[slot] = t;
      }
      __syncthreads();
      R a0x = R(0), a0y = R(0), a0z = R(0), a1x = R(0), a1y = R(0), a1z = R(0);
      if (!core_law) {
#pragma unroll 8
        for (int k = 0; k < T; ++k) {
          V4 q = tile[k];
          R dx0 = q.x - x0, dy0 = q.y - y0, dz0 = q.z - z0;
          R dx1 = q.x - x1, dy1 = q.y - y1, dz1 = q.z - z1;
          R s20 = fma(dx0, dx0, fma(dy0, dy0, fma(dz0, dz0, eps2)));
          R s21 = fma(dx1, dx1, fma(dy1, dy1, fma(dz1, dz1, eps2)));
          R i0 = rsqrt_r<R>(s20), i1 = rsqrt_r<R>(s21);
          R s0 = q.w * (i0 * i0 * i0), s1 = q.w * (i1 * i1 * i1);
          a0x = fma(dx0, s0, a0x); a0y = fma(dy0, s0, a0y); a0z = fma(dz0, s0, a0z);
          a1x = fma(dx1, s1, a1x); a1y = fma(dy1, s1, a1y); a1z = fma(dz1, s1, a1z);
        }
      } else {
#pragma unroll 4
        for (int k = 0; k < T; ++k) {
          V4 q = tile[k];
          const int jg = base + k;
          // core radius of the higher-slot body (gravity.rs:126-131); coincident bodies exert
          // nothing (|d| < 1e-9, gravity.rs:119-122)
          {
            R dx = q.x - x0, dy = q.y - y0, dz = q.z - z0;
            R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
            bool j_hi = jg > il0;
            R sz2 = j_hi ? tsz2[k] : sz2_0;
            R isz3 = j_hi ? tisz3[k] : isz3_0;
            R inv = rsqrt_r<R>(r2);
            R sd = (r2 >= sz2) ? inv * inv * inv : isz3;
            R s = (r2 < R(1e-18)) ? R(0) : q.w * sd;
            a0x = fma(dx, s, a0x); a0y = fma(dy, s, a0y); a0z = fma(dz, s, a0z);
          }
          {
            R dx = q.x - x1, dy = q.y - y1, dz = q.z - z1;
            R r2 = fma(dx, dx, fma(dy, dy, dz * dz));
            bool j_hi = jg > il1;
            R sz2 = j_hi ? tsz2[k] : sz2_1;
            R isz3 = j_hi ? tisz3[k] : isz3_1;
            R inv = rsqrt_r<R>(r2);
            R sd = (r2 >= sz2) ? inv * inv * inv : isz3;
            R s = (r2 < R(1e-18)) ? R(0) : q.w * sd;
            a1x = fma(dx, s, a1x); a1y = fma(dy, s, a1y); a1z = fma(dz, s, a1z);
          }
        }
      }
      da0x += double(a0x); da0y += double(a0y); da0z += double(a0z);
      da1x += double(a1x); da1y += double(a1y); da1z += double(a1z);
      __syncthreads();
    }
    double* p = partial + g.out_off;
    if (v0) { p[il0] = da0x; p[g.n + il0] = da0y; p[2 * (size_t)g.n + il0] = da0z; }
    if (v1) { p[il1] = da1x; p[g.n + il1] = da1y; p[2 * (size_t)g.n + il1] = da1z; }
  }
}

// Mixed path: one warp owns an i-tile (thread t: bodies i0 + t + 32h, h = 0..3). The four
// i-bodies form two pairs, and the Plummer pair terms run as packed FP32x2 instructions (one
// instruction, two lanes of arithmetic): the j-body is staged in shared memory already duplicated
// ({x,x,y,y}, {z,z,m,m}) so that both halves of a pair read it with no register moves. Each pair
// term is rounded exactly as the scalar form fma(dx,dx,fma(dy,dy,fma(dz,dz,eps2))), m*((i*i)*i),
// fma(dx,s,acc) would round it. The size-core law keeps the scalar form.
constexpr int kMixKI = 4;
constexpr int kMixThreads = kGravTile / kMixKI;

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// The PTX ISA's approximate reciprocal square root with subnormals flushed: one MUFU operation and
// nothing else. (The non-flushing form adds a range fix-up around it on the FMA pipe, which is the
// pipe that bounds this kernel.) Pair distances here are never subnormal: the Plummer law adds
// eps^2 > 0, and the size-core law discards r^2 < 1e-18.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// COMP (the MIXED precision): positions relative to the tile reference are carried as FP32 pairs
// hi + lo (the remainder of the FP64 difference), and a pair's difference is (hi_j - hi_i) +
// (lo_j - lo_i): the first term is exact for nearby bodies (Sterbenz), so a close pair's
// separation is accurate to FP32 rounding of the separation itself rather than of the distance to
// the tile reference. Without it (MIXED_FAST) a close pair far from the reference carries that
// reference distance's rounding, which dense clusters amplify over many steps.
template <bool COMP>
__global__ void __launch_bounds__(kMixThreads) k_gravity_items_mixed(const double4* __restrict__ pm,
                                                                     const double* __restrict__ size,
                                                                     const GravItem* __restrict__ items, int n_items,
                                                                     int* __restrict__ head,
                                                                     double* __restrict__ partial,
                                                                     const int* __restrict__ world_of_body,
                                                                     const int* __restrict__ w_active) {
  constexpr int T = kGravTile;
  constexpr int H = kMixThreads;
  __shared__ float4 tq[T][COMP ? 3 : 2];
  __shared__ float tsz2[T];
  __shared__ float tisz3[T];
  __shared__ int cur;
  for (;;) {
    if (threadIdx.x == 0) cur = atomicAdd(head, 1);
    __syncthreads();
    const int it = cur;
    __syncthreads();
    if (it >= n_items) return;
    const GravItem g = items[it];
    if (w_active && !w_active[world_of_body[g.body_off]]) continue;  // the world holds this step
    const double4* wpm = pm + g.body_off;
    const double4 c = wpm[g.i0];
    const bool core_law = g.law == EXG_GRAVITY_SIZE_CORE;
    int il[kMixKI];
    bool v[kMixKI];
    float px[kMixKI], py[kMixKI], pz[kMixKI], sz2[kMixKI], isz3[kMixKI];
    float lx[kMixKI], ly[kMixKI], lz[kMixKI];
#pragma unroll
    for (int h = 0; h < kMixKI; ++h) {
      il[h] = g.i0 + threadIdx.x + h * H;
      v[h] = il[h] < g.n;
      const double4 p = v[h] ? wpm[il[h]] : c;
      const double rx = p.x - c.x, ry = p.y - c.y, rz = p.z - c.z;
      px[h] = float(rx);
      py[h] = float(ry);
      pz[h] = float(rz);
      lx[h] = COMP ? float(rx - double(px[h])) : 0.f;
      ly[h] = COMP ? float(ry - double(py[h])) : 0.f;
      lz[h] = COMP ? float(rz - double(pz[h])) : 0.f;
      sz2[h] = 0.f;
      isz3[h] = 0.f;
      if (core_law && v[h]) {
        const double sd = size[g.body_off + il[h]];
        sz2[h] = float(sd * sd);
        isz3[h] = float(1.0 / (sd * sd * sd));
      }
    }
    const float2 nxA = f2(-px[0], -px[1]), nyA = f2(-py[0], -py[1]), nzA = f2(-pz[0], -pz[1]);
    const float2 nxB = f2(-px[2], -px[3]), nyB = f2(-py[2], -py[3]), nzB = f2(-pz[2], -pz[3]);
    const float2 mxA = f2(-lx[0], -lx[1]), myA = f2(-ly[0], -ly[1]), mzA = f2(-lz[0], -lz[1]);
    const float2 mxB = f2(-lx[2], -lx[3]), myB = f2(-ly[2], -ly[3]), mzB = f2(-lz[2], -lz[3]);
    const float e2 = float(g.eps2);
    const float2 eps2 = f2(e2, e2);
    double acc[kMixKI][3];
#pragma unroll
    for (int h = 0; h < kMixKI; ++h) acc[h][0] = acc[h][1] = acc[h][2] = 0.0;
    for (int base = g.j0; base < g.j1; base += T) {
#pragma unroll
      for (int h = 0; h < kMixKI; ++h) {
        const int slot = threadIdx.x + h * H;
        const int j = base + slot;
        float x = 0.f, y = 0.f, z = 0.f, m = 0.f, xl = 0.f, yl = 0.f, zl = 0.f;
        if (j < g.j1) {
          const double4 q = wpm[j];
          const double rx = q.x - c.x, ry = q.y - c.y, rz = q.z - c.z;
          x = float(rx);
          y = float(ry);
          z = float(rz);
          if (COMP) {
            xl = float(rx - double(x));
            yl = float(ry - double(y));
            zl = float(rz - double(z));
          }
          m = float(q.w);
          if (core_law) {
            const double sd = size[g.body_off + j];
            tsz2[slot] = float(sd * sd);
            tisz3[slot] = float(1.0 / (sd * sd * sd));
          }
        } else if (core_law) {
          tsz2[slot] = 1.f;
          tisz3[slot] = 0.f;
        }
        tq[slot][0] = make_float4(x, x, y, y);
        tq[slot][1] = make_float4(z, z, m, m);
        if (COMP) tq[slot][COMP ? 2 : 0] = make_float4(xl, yl, zl, 0.f);
      }
      __syncthreads();
      float a[kMixKI][3];
      if (!core_law) {
        float2 axA = f2(0.f, 0.f), ayA = axA, azA = axA, axB = axA, ayB = axA, azB = axA;
#pragma unroll 4
        for (int k = 0; k < T; ++k) {
          const float4 u = tq[k][0], w = tq[k][1];
          const float2 qx = f2(u.x, u.y), qy = f2(u.z, u.w), qz = f2(w.x, w.y), qm = f2(w.z, w.w);
          float2 dxA = __fadd2_rn(qx, nxA), dyA = __fadd2_rn(qy, nyA), dzA = __fadd2_rn(qz, nzA);
          float2 dxB = __fadd2_rn(qx, nxB), dyB = __fadd2_rn(qy, nyB), dzB = __fadd2_rn(qz, nzB);
          if (COMP) {  // add the difference of the remainders
            const float4 l = tq[k][COMP ? 2 : 0];
            const float2 lxj = f2(l.x, l.x), lyj = f2(l.y, l.y), lzj = f2(l.z, l.z);
            dxA = __fadd2_rn(dxA, __fadd2_rn(lxj, mxA));
            dyA = __fadd2_rn(dyA, __fadd2_rn(lyj, myA));
            dzA = __fadd2_rn(dzA, __fadd2_rn(lzj, mzA));
            dxB = __fadd2_rn(dxB, __fadd2_rn(lxj, mxB));
            dyB = __fadd2_rn(dyB, __fadd2_rn(lyj, myB));
            dzB = __fadd2_rn(dzB, __fadd2_rn(lzj, mzB));
          }
          const float2 rA = __ffma2_rn(dxA, dxA, __ffma2_rn(dyA, dyA, __ffma2_rn(dzA, dzA, eps2)));
          const float2 rB = __ffma2_rn(dxB, dxB, __ffma2_rn(dyB, dyB, __ffma2_rn(dzB, dzB, eps2)));
          const float2 iA = f2(rsqrt_ftz(rA.x), rsqrt_ftz(rA.y)), iB = f2(rsqrt_ftz(rB.x), rsqrt_ftz(rB.y));
          const float2 sA = __fmul2_rn(qm, __fmul2_rn(__fmul2_rn(iA, iA), iA));
          const float2 sB = __fmul2_rn(qm, __fmul2_rn(__fmul2_rn(iB, iB), iB));
          axA = __ffma2_rn(dxA, sA, axA); ayA = __ffma2_rn(dyA, sA, ayA); azA = __ffma2_rn(dzA, sA, azA);
          axB = __ffma2_rn(dxB, sB, axB); ayB = __ffma2_rn(dyB, sB, ayB); azB = __ffma2_rn(dzB, sB, azB);
        }
        a[0][0] = axA.x; a[1][0] = axA.y; a[2][0] = axB.x; a[3][0] = axB.y;
        a[0][1] = ayA.x; a[1][1] = ayA.y; a[2][1] = ayB.x; a[3][1] = ayB.y;
        a[0][2] = azA.x; a[1][2] = azA.y; a[2][2] = azB.x; a[3][2] = azB.y;
      } else {
#pragma unroll
        for (int h = 0; h < kMixKI; ++h) a[h][0] = a[h][1] = a[h][2] = 0.f;
#pragma unroll 2
        for (int k = 0; k < T; ++k) {
          const float4 u = tq[k][0], w = tq[k][1];
          const int jg = base + k;
          const float ts2 = tsz2[k], tis3 = tisz3[k];
#pragma unroll
          for (int h = 0; h < kMixKI; ++h) {
            // core radius of the higher-slot body (gravity.rs:126-131); coincident bodies exert
            // nothing (|d| < 1e-9, gravity.rs:119-122)
            float dx = u.x - px[h], dy = u.z - py[h], dz = w.x - pz[h];
            if (COMP) {
              const float4 l = tq[k][COMP ? 2 : 0];
              dx = dx + (l.x - lx[h]);
              dy = dy + (l.y - ly[h]);
              dz = dz + (l.z - lz[h]);
            }
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool j_hi = jg > il[h];
            const float s2 = j_hi ? ts2 : sz2[h];
            const float i3 = j_hi ? tis3 : isz3[h];
            const float inv = rsqrt_ftz(r2);
            const float sd = (r2 >= s2) ? inv * inv * inv : i3;
            const float sc = (r2 < 1e-18f) ? 0.f : w.z * sd;
            a[h][0] = fmaf(dx, sc, a[h][0]);
            a[h][1] = fmaf(dy, sc, a[h][1]);
            a[h][2] = fmaf(dz, sc, a[h][2]);
          }
        }
      }
#pragma unroll
      for (int h = 0; h < kMixKI; ++h) {
        acc[h][0] += double(a[h][0]);
        acc[h][1] += double(a[h][1]);
        acc[h][2] += double(a[h][2]);
      }
      __syncthreads();
    }
    double* out = partial + g.out_off;
#pragma unroll
    for (int h = 0; h < kMixKI; ++h)
      if (v[h]) {
        out[il[h]] = acc[h][0];
        out[g.n + il[h]] = acc[h][1];
        out[2 * (size_t)g.n + il[h]] = acc[h][2];
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
                         int* head, int precision, double* partial, cudaStream_t s, const int* world_of_body,
                         const int* w_active) {
  if (n_items <= 0) return EXG_OK;
  EXG_CUDA_TRY(cudaMemsetAsync(head, 0, sizeof(int), s));
  int sms = dev->sm_count > 0 ? dev->sm_count : 148;
  const double4* pm = reinterpret_cast<const double4*>(pos_mass);
  int tok = prof_begin(dev, PROF_GRAVITY, s);
  if (precision == EXG_PRECISION_MIXED)
    k_gravity_items_mixed<true><<<std::min(n_items, sms * std::max(1, dev->tune_gravity_ctas_per_sm.load())), kMixThreads, 0, s>>>(pm, size, items, n_items, head, partial,
                                                                             world_of_body, w_active);
  else if (precision == EXG_PRECISION_MIXED_FAST)
    k_gravity_items_mixed<false><<<std::min(n_items, sms * std::max(1, dev->tune_gravity_ctas_per_sm.load())), kMixThreads, 0, s>>>(pm, size, items, n_items, head, partial,
                                                                             world_of_body, w_active);
  else
    k_gravity_items<double><<<std::min(n_items, sms * 16), kGravThreads, 0, s>>>(pm, size, items, n_items, head,
                                                                                partial, world_of_body, w_active);
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

// A new device handle looks the address up again on its first no-allocation call, so a context
// the host re-created on that device (after cudaDeviceReset) is not served a stale address.
void exg_internal_noalloc_forget(int ordinal) {
  if (ordinal < 0 || ordinal >= 256) return;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  g_noalloc_addr[ordinal] = nullptr;
}

extern "C" int exg_gravity_forces_noalloc(exg_device_t dev, const double* d_pos_mass, const double* d_size, int32_t n,
                                          int32_t law, double G, double softening, int32_t precision, double* d_force) {
  if (!dev || n < 0 || (n > 0 && (!d_pos_mass || !d_force))) return EXG_ERR_INVALID_ARGUMENT;
  if (n > EXG_NOALLOC_MAX_BODIES) return EXG_ERR_INVALID_ARGUMENT;
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
