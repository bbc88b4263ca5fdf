// Implicit mid-point Newton step on the device; see world_newton.cuh for the structure.
//
// Per island, one CTA executes Newton::solve_step (crates/newton/src/integrator/implicit/newton.rs:543-683):
//   span loop over dt / 2^depth (MAX_DEPTH 8, the log2 stiffness signal moves the depth),
//   newton_solve (:334-530): up to max_newton iterations of
//     PRE (functions::pre) -> joint value + Jacobian -> gather + POST (functions::body_post)
//     -> worst relative residual (:139-151) -> assembly (rows/assemble.rs) -> linear solve
//     -> backtracking line search over the fractions 1, 1/2, ..., 1/128, first decrease wins
//   commit_span (:708-753): M = M0 * exp(span v), P = 2 P_mid - P_n (implicit Euler if the span
//   did not converge).
// The linear solve is exact block elimination on the island's tree (leaves to root, then back
// substitution) instead of the reference's dense Newton-Schulz iteration on m^2 blocks: both
// solve the same Newton system, so the converged iterate is the same; the tree solve is O(m).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <new>
#include "body.cuh"
#include "joint_eval.cuh"
#include "world_newton.cuh"

namespace {

using namespace exg;

#ifndef EXG_NEWTON_MIN_BLOCKS
#define EXG_NEWTON_MIN_BLOCKS 1  // CTAs per SM the register budget is sized for
#endif
#ifndef EXG_NEWTON_THREADS
#define EXG_NEWTON_THREADS 256
#endif
constexpr int kThreads = EXG_NEWTON_THREADS;
constexpr int kMinBlocks = EXG_NEWTON_MIN_BLOCKS;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxDepth = 8;
constexpr int kThresholdLog2 = 8;
constexpr int kPerHalvingLog2 = 4;
constexpr double kHuge = 1e9;
constexpr double kFloor2 = 1e-9 * 1e-9;
constexpr int kJacStride = 42;  // per (joint, slice): value[6] + d[36]

struct Scratch {
  double *vm, *base, *best, *trial, *mid, *snap, *ext, *conn, *jac, *mass, *mass0, *rhs, *scale, *D, *Dinv, *Acp, *Apc, *S,
      *bvec, *dv;
};

EXG_HD long long scratch_doubles(int nb, int nj, int m) {
  return (long long)nb * (6 * 4 + 8 + 6 * 2) + (long long)nj * (6 + 4 * kJacStride) + (long long)m * (36 * 7 + 6 * 3 + 2);
}

__device__ Scratch carve(double* p, int nb, int nj, int m) {
  Scratch s;
  s.vm = p; p += nb * 6;
  s.base = p; p += nb * 6;
  s.best = p; p += nb * 6;
  s.trial = p; p += nb * 6;
  s.mid = p; p += nb * 8;
  s.snap = p; p += nb * 6;
  s.ext = p; p += nb * 6;
  s.conn = p; p += (size_t)nj * 6;
  s.jac = p; p += (size_t)nj * 4 * kJacStride;
  s.mass = p; p += (size_t)m * 36;
  s.mass0 = p; p += (size_t)m * 36;
  s.rhs = p; p += (size_t)m * 6;
  s.scale = p; p += (size_t)m * 2;
  s.D = p; p += (size_t)m * 36;
  s.Dinv = p; p += (size_t)m * 36;
  s.Acp = p; p += (size_t)m * 36;
  s.Apc = p; p += (size_t)m * 36;
  s.S = p; p += (size_t)m * 36;
  s.bvec = p; p += (size_t)m * 6;
  s.dv = p; p += (size_t)m * 6;
  return s;
}

struct WorldRef {
  double* pose;
  double* mom;
  const double* mass;
  const double* inertia;
  const int* kinematic;
  const int* diagonal;
  const double* pos_mass;
  const double* grav_partial;
  const exg_step_params_t* wparams;
  const long long* w_poff;
  const int* w_splits;
  const int* w_n;
  const int* w_body_off;
  const int* w_active;
  int n;
};

// The island's world parameters, resolved once per island.
struct IslandParams {
  double dt, warp, tol2, G, pose_factor_scale;
  int max_newton;
  int splits, nw, wbody_off;
  const double* part;
};

struct Ctx {
  NewtonDeviceArrays A;
  IslandDesc d;
  WorldRef W;
  IslandParams P;
  Scratch s;
  int island;
  EXG_HD int gbody(int q) const { return A.isl_body[d.body_off + q]; }
};

// Phase timer: thread 0 accumulates SM clock cycles between phase boundaries (all threads have
// passed a barrier there) into shared counters; the CTA adds them to the global totals at the end.
struct PhaseTimer {
  long long* acc;  // shared [kPhases]
  long long t0;
  __device__ void start() { if (threadIdx.x == 0) t0 = clock64(); }
  __device__ void lap(int phase) {
    if (threadIdx.x == 0) {
      long long t = clock64();
      acc[phase] += t - t0;
      t0 = t;
    }
  }
};

// ── block-wide reductions ───────────────────────────────────────────────────
__device__ double nan_max(double a, double b) {
  if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000ULL);
  return a > b ? a : b;
}
__device__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = nan_max(v, __shfl_xor_sync(0xffffffffu, v, o));
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = red[0];
  for (int k = 1; k < kWarps; ++k) r = nan_max(r, red[k]);
  __syncthreads();
  return r;
}
__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = red[0];
  for (int k = 1; k < kWarps; ++k) r += red[k];
  __syncthreads();
  return r;
}

// ── phases ──────────────────────────────────────────────────────────────────
// PRE: mid = exp(half/2 v) * pose for every island body (functions::pre)
__device__ void phase_pre(const Ctx& c, const double* v, double half) {
  for (int q = threadIdx.x; q < c.d.nb; q += blockDim.x) {
    int g = c.gbody(q);
    double pose[8], vb[6], e[8], m[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) pose[k] = c.W.pose[(size_t)k * c.W.n + g];
    screw_from6(v + 6 * q, vb);
    twist_exp(vb, half, e);
    motor_compose(pose, e, m);
#pragma unroll
    for (int k = 0; k < 8; ++k) c.s.mid[8 * q + k] = m[k];
  }
}

// Joint values (and Jacobian slices) at (mid, v): conn[q] = wrench on end a. MIXED evaluates the
// derivative slices in FP32 duals; the values that enter the residual always come from an FP64
// evaluation, so the converged iterate is an FP64 solution whatever the Jacobian's precision.
template <bool MIXED>
__device__ void phase_joints(const Ctx& c, const double* v, bool jac) {
  const int nj = c.d.nj;
  const int joff = c.d.joint_off;
  if (jac) {
    for (int t = threadIdx.x; t < 4 * nj; t += blockDim.x) {
      int q = t >> 2, slice = t & 3;
      int a = c.A.jl_a[joff + q], b = c.A.jl_b[joff + q];
      const int law = c.A.jl_law[joff + q];
      const double* prm = c.A.jl_params + 10 * (size_t)(joff + q);
      double* o = c.s.jac + ((size_t)q * 4 + slice) * kJacStride;
      if (MIXED) {
        float pa[8], pb[8], va[6], vb[6], val[6], dd[36];
#pragma unroll
        for (int k = 0; k < 8; ++k) { pa[k] = float(c.s.mid[8 * a + k]); pb[k] = float(c.s.mid[8 * b + k]); }
#pragma unroll
        for (int k = 0; k < 6; ++k) { va[k] = float(v[6 * a + k]); vb[k] = float(v[6 * b + k]); }
        joint_jacobian_slice<float>(law, prm, pa, pb, va, vb, c.P.dt, c.P.warp, slice, val, dd);
#pragma unroll
        for (int r = 0; r < 6; ++r) o[r] = double(val[r]);
#pragma unroll
        for (int k = 0; k < 36; ++k) o[6 + k] = double(dd[k]);
        if (slice == 0) {
          double out[12];
          joint_plain<double>(law, prm, c.s.mid + 8 * a, c.s.mid + 8 * b, v + 6 * a, v + 6 * b, c.P.dt, c.P.warp, out);
#pragma unroll
          for (int r = 0; r < 6; ++r) c.s.conn[6 * q + r] = out[r];
        }
      } else {
        double val[6], dd[36];
        joint_jacobian_slice<double>(law, prm, c.s.mid + 8 * a, c.s.mid + 8 * b, v + 6 * a, v + 6 * b, c.P.dt, c.P.warp,
                                     slice, val, dd);
#pragma unroll
        for (int r = 0; r < 6; ++r) o[r] = val[r];
#pragma unroll
        for (int k = 0; k < 36; ++k) o[6 + k] = dd[k];
        if (slice == 0) {
#pragma unroll
          for (int r = 0; r < 6; ++r) c.s.conn[6 * q + r] = val[r];
        }
      }
    }
  } else {
    for (int q = threadIdx.x; q < nj; q += blockDim.x) {
      int a = c.A.jl_a[joff + q], b = c.A.jl_b[joff + q];
      double out[12];
      joint_plain<double>(c.A.jl_law[joff + q], c.A.jl_params + 10 * (size_t)(joff + q), c.s.mid + 8 * a, c.s.mid + 8 * b,
                          v + 6 * a, v + 6 * b, c.P.dt, c.P.warp, out);
#pragma unroll
      for (int r = 0; r < 6; ++r) c.s.conn[6 * q + r] = out[r];
    }
  }
}

// Gather + POST for every dynamic node; returns the worst relative residual^2 (newton.rs:139-151).
__device__ double phase_post(const Ctx& c, const double* v, double half, double* red) {
  double worst = 0.0;
  for (int i = threadIdx.x; i < c.d.m; i += blockDim.x) {
    int q = c.A.dn_body[c.d.dyn_off + i];
    int g = c.gbody(q);
    double tot[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) tot[k] = c.s.ext[6 * q + k];
    int p0 = c.A.ib_inc_ptr[c.d.inc_off + q], p1 = c.A.ib_inc_ptr[c.d.inc_off + q + 1];
    for (int t = p0; t < p1; ++t) {
      int ref = c.A.ib_inc_ref[t];
      int jq = ref >> 1;
      if (ref & 1) {
#pragma unroll
        for (int k = 0; k < 6; ++k) tot[k] = tot[k] - c.s.conn[6 * jq + k];
      } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) tot[k] = tot[k] + c.s.conn[6 * jq + k];
      }
    }
    double I9[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) I9[k] = c.W.inertia[(size_t)k * c.W.n + g];
    const bool diag = c.W.diagonal[g] != 0;
    const double mass = c.W.mass[g];
    const double* mid = c.s.mid + 8 * q;
    double inv[8];
    motor_reverse(mid, inv);
    double* blk = c.s.mass + 36 * (size_t)i;
#pragma unroll
    for (int col = 0; col < 6; ++col) {
      double e6[6] = {0, 0, 0, 0, 0, 0};
      e6[col] = 1.0;
      double eb[6], ebody[6], b6[6], wv[6], p6[6], pb[6], cw[6], c6[6];
      screw_from6(e6, eb);
      twist_transport(eb, inv, ebody);
      screw_to6(ebody, b6);
      wv[0] = b6[0]; wv[1] = b6[1]; wv[2] = b6[2]; wv[3] = b6[3]; wv[4] = b6[4]; wv[5] = b6[5];
      inertia_apply(I9, diag, false, mass, wv, p6);
      screw_from6(p6, pb);
      wrench_transport(pb, mid, cw);
      screw_to6(cw, c6);
#pragma unroll
      for (int r = 0; r < 6; ++r) blk[r * 6 + col] = c6[r];
    }
    const double* vv = v + 6 * q;
    double p[6], nn[6], hh[6], res[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) acc += blk[r * 6 + k] * vv[k];
      p[r] = acc;
      nn[r] = c.s.snap[6 * q + r];
      hh[r] = tot[r] * half;
    }
#pragma unroll
    for (int r = 0; r < 6; ++r) res[r] = -(p[r] - nn[r] - hh[r]);
#pragma unroll
    for (int r = 0; r < 6; ++r) c.s.rhs[6 * i + r] = res[r];
    auto sq3 = [](const double* x) { return x[0] * x[0] + x[1] * x[1] + x[2] * x[2]; };
    double lin = fmax(fmax(fmax(sq3(p), sq3(nn)), sq3(hh)), kFloor2);
    double ang = fmax(fmax(fmax(sq3(p + 3), sq3(nn + 3)), sq3(hh + 3)), kFloor2);
    c.s.scale[2 * i] = lin;
    c.s.scale[2 * i + 1] = ang;
    worst = nan_max(worst, sq3(res) / lin);
    worst = nan_max(worst, sq3(res + 3) / ang);
  }
  return block_max(worst, red);
}

__device__ void copy_mass0(const Ctx& c) {
  for (int t = threadIdx.x; t < 36 * c.d.m; t += blockDim.x) c.s.mass0[t] = c.s.mass[t];
}

// Assembly (rows/assemble.rs, functions::assemble_term): per target block and entry, the
// mass block (diagonal only) then every contributing joint end in joint order with the
// midpoint factors pf = -half^2 on pose columns and vf = -half on velocity columns.
// Returns ||A||_F^2.
__device__ double phase_assemble(const Ctx& c, double half, double* red) {
  const double pf = -(half * half) * c.P.pose_factor_scale, vf = -half;
  double sumsq = 0.0;
  const int cells = 3 * c.d.m;
  for (int t = threadIdx.x; t < cells * 36; t += blockDim.x) {
    int cell = t / 36, e = t % 36;
    int i = cell / 3, kind = cell % 3;
    int r = e / 6, col = e % 6;
    double acc = (kind == 0) ? c.s.mass0[36 * (size_t)i + e] : 0.0;
    int p0 = c.A.cell_ptr[c.d.cell_off + cell], p1 = c.A.cell_ptr[c.d.cell_off + cell + 1];
    for (int k = p0; k < p1; ++k) {
      int term = c.A.cell_terms[k];
      int q = term >> 2, re = (term >> 1) & 1, ce = term & 1;
      const double* jp = c.s.jac + ((size_t)q * 4 + ce) * kJacStride + 6;
      const double* jv = c.s.jac + ((size_t)q * 4 + 2 + ce) * kJacStride + 6;
      double pv = jp[r * 6 + col], vv = jv[r * 6 + col];
      if (re) { pv = -pv; vv = -vv; }
      acc = acc + pf * pv + vf * vv;
    }
    double* dst = kind == 0 ? c.s.D : (kind == 1 ? c.s.Acp : c.s.Apc);
    dst[36 * (size_t)i + e] = acc;
    if (kind == 0 || c.A.dn_parent[c.d.dyn_off + i] >= 0) sumsq += acc * acc;
  }
  return block_sum(sumsq, red);
}

// Warp-cooperative 6x6 inverse by Gauss-Jordan with partial pivoting: lane c < 12 holds
// column c of [A | I]. Returns false (to every lane) if a pivot is zero or not finite.
__device__ bool warp_inverse6(const double* a, double* out) {
  const int lane = threadIdx.x & 31;
  double col[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    if (lane < 6) col[r] = a[r * 6 + lane];
    else col[r] = (lane - 6 == r) ? 1.0 : 0.0;
  }
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    int piv = k;
    double best = fabs(col[k]);
#pragma unroll
    for (int r = k + 1; r < 6; ++r) {
      double x = fabs(col[r]);
      if (x > best) { best = x; piv = r; }
    }
    piv = __shfl_sync(0xffffffffu, piv, k);
    double tk = col[k], tp = col[k];
#pragma unroll
    for (int r = k; r < 6; ++r) if (r == piv) tp = col[r];
#pragma unroll
    for (int r = k; r < 6; ++r) if (r == piv) col[r] = tk;
    col[k] = tp;
    double pv = __shfl_sync(0xffffffffu, col[k], k);
    if (!(fabs(pv) > 0.0) || !isfinite(pv)) ok = false;
    double ip = 1.0 / pv;
    col[k] = col[k] * ip;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (r == k) continue;
      double f = __shfl_sync(0xffffffffu, col[r], k);
      col[r] = col[r] - f * col[k];
    }
  }
  if (lane >= 6 && lane < 12) {
#pragma unroll
    for (int r = 0; r < 6; ++r) out[r * 6 + (lane - 6)] = col[r];
  }
  __syncwarp();
  return ok;
}

// C = A * B (6x6, row-major) or C -= A * B, computed by one warp.
template <bool Sub>
__device__ void warp_mm6(const double* A, const double* B, double* C) {
  const int lane = threadIdx.x & 31;
  double v0 = 0.0, v1 = 0.0;
  int e0 = lane, e1 = lane + 32;
  {
    int r = e0 / 6, cc = e0 % 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) v0 += A[r * 6 + k] * B[k * 6 + cc];
  }
  if (e1 < 36) {
    int r = e1 / 6, cc = e1 % 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) v1 += A[r * 6 + k] * B[k * 6 + cc];
  }
  __syncwarp();
  if (Sub) {
    C[e0] = C[e0] - v0;
    if (e1 < 36) C[e1] = C[e1] - v1;
  } else {
    C[e0] = v0;
    if (e1 < 36) C[e1] = v1;
  }
  __syncwarp();
}
// y -= A x (6x6 * 6) by one warp (lanes 0..5)
__device__ void warp_mv6_sub(const double* A, const double* x, double* y) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  if (lane < 6) {
#pragma unroll
    for (int k = 0; k < 6; ++k) s += A[lane * 6 + k] * x[k];
  }
  __syncwarp();
  if (lane < 6) y[lane] = y[lane] - s;
  __syncwarp();
}
__device__ void warp_mv6(const double* A, const double* x, double* y) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  if (lane < 6) {
#pragma unroll
    for (int k = 0; k < 6; ++k) s += A[lane * 6 + k] * x[k];
  }
  __syncwarp();
  if (lane < 6) y[lane] = s;
  __syncwarp();
}

// Exact solve of A dv = rhs on the island's elimination forest. Returns false if a pivot
// block is singular (dv is then NaN, which the line search rejects).
__device__ bool phase_solve(const Ctx& c, int* flag) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = c.d.m;
  const int* lv = c.A.lv_ptr + c.d.lv_off;
  const int* nodes = c.A.lv_nodes + c.d.dyn_off;
  const int* par = c.A.dn_parent + c.d.dyn_off;
  const int* chp = c.A.ch_ptr + c.d.dyn_off;  // absolute offsets into ch_idx
  const int* chi = c.A.ch_idx;
  if (threadIdx.x == 0) *flag = 1;
  for (int t = threadIdx.x; t < 6 * m; t += blockDim.x) c.s.bvec[t] = c.s.rhs[t];
  __syncthreads();
  for (int L = c.d.n_levels - 1; L >= 1; --L) {
    for (int k = lv[L] + warp; k < lv[L + 1]; k += kWarps) {
      int i = nodes[k];
      bool ok = warp_inverse6(c.s.D + 36 * (size_t)i, c.s.Dinv + 36 * (size_t)i);
      if (!ok && lane == 0) *flag = 0;
      warp_mm6<false>(c.s.Apc + 36 * (size_t)i, c.s.Dinv + 36 * (size_t)i, c.s.S + 36 * (size_t)i);
    }
    __syncthreads();
    for (int k = lv[L - 1] + warp; k < lv[L]; k += kWarps) {
      int p = nodes[k];
      for (int t = chp[p]; t < chp[p + 1]; ++t) {
        int ch = chi[t];
        warp_mm6<true>(c.s.S + 36 * (size_t)ch, c.s.Acp + 36 * (size_t)ch, c.s.D + 36 * (size_t)p);
        warp_mv6_sub(c.s.S + 36 * (size_t)ch, c.s.bvec + 6 * ch, c.s.bvec + 6 * p);
      }
    }
    __syncthreads();
  }
  for (int k = lv[0] + warp; k < lv[1]; k += kWarps) {
    int i = nodes[k];
    bool ok = warp_inverse6(c.s.D + 36 * (size_t)i, c.s.Dinv + 36 * (size_t)i);
    if (!ok && lane == 0) *flag = 0;
    warp_mv6(c.s.Dinv + 36 * (size_t)i, c.s.bvec + 6 * i, c.s.dv + 6 * i);
  }
  __syncthreads();
  for (int L = 1; L < c.d.n_levels; ++L) {
    for (int k = lv[L] + warp; k < lv[L + 1]; k += kWarps) {
      int i = nodes[k];
      int p = par[i];
      warp_mv6_sub(c.s.Acp + 36 * (size_t)i, c.s.dv + 6 * p, c.s.bvec + 6 * i);
      warp_mv6(c.s.Dinv + 36 * (size_t)i, c.s.bvec + 6 * i, c.s.dv + 6 * i);
    }
    __syncthreads();
  }
  bool ok = *flag != 0;
  __syncthreads();
  if (!ok) {
    for (int t = threadIdx.x; t < 6 * m; t += blockDim.x) c.s.dv[t] = __longlong_as_double(0x7ff8000000000000ULL);
    __syncthreads();
  }
  return ok;
}

__device__ void copy_bodies6(const Ctx& c, const double* src, double* dst) {
  for (int t = threadIdx.x; t < 6 * c.d.nb; t += blockDim.x) dst[t] = src[t];
}

// trial = base + alpha dv on the dynamic bodies; kinematic bodies keep their prescribed twist.
__device__ void make_trial(const Ctx& c, double alpha) {
  for (int t = threadIdx.x; t < 6 * c.d.nb; t += blockDim.x) {
    int q = t / 6, k = t % 6;
    int i = c.A.ib_order[c.d.body_off + q];
    c.s.trial[t] = (i >= 0) ? c.s.base[t] + c.s.dv[6 * i + k] * alpha : c.s.base[t];
  }
}

// world twist and world momentum of every island body at the current state
__device__ void load_world_state(const Ctx& c) {
  for (int q = threadIdx.x; q < c.d.nb; q += blockDim.x) {
    int g = c.gbody(q);
    double pose[8], mom[6], I9[9];
#pragma unroll
    for (int k = 0; k < 8; ++k) pose[k] = c.W.pose[(size_t)k * c.W.n + g];
#pragma unroll
    for (int k = 0; k < 6; ++k) mom[k] = c.W.mom[(size_t)k * c.W.n + g];
#pragma unroll
    for (int k = 0; k < 9; ++k) I9[k] = c.W.inertia[(size_t)k * c.W.n + g];
    bool kin = c.W.kinematic[g] != 0;
    double wv[6];
    world_velocity(pose, mom, I9, c.W.diagonal[g] != 0, kin, c.W.mass[g], wv);
    double mb[6], pw[6], p6[6];
    screw_from6(mom, mb);
    wrench_transport(mb, pose, pw);
    screw_to6(pw, p6);
#pragma unroll
    for (int k = 0; k < 6; ++k) { c.s.vm[6 * q + k] = wv[k]; c.s.snap[6 * q + k] = p6[k]; }
  }
}

// external wrench per island body: gravity (F, p x F) frozen over the whole step
__device__ void load_external(const Ctx& c) {
  for (int q = threadIdx.x; q < c.d.nb; q += blockDim.x) {
    double* e = c.s.ext + 6 * q;
#pragma unroll
    for (int k = 0; k < 6; ++k) e[k] = 0.0;
    if (c.P.splits <= 0) continue;
    int g = c.gbody(q);
    int il = g - c.P.wbody_off;
    double4 pm = reinterpret_cast<const double4*>(c.W.pos_mass)[g];
    double f[3];
    for (int k = 0; k < 3; ++k) {
      double acc = 0.0;
      for (int s = 0; s < c.P.splits; ++s) acc += c.P.part[(size_t)s * 3 * c.P.nw + (size_t)k * c.P.nw + il];
      f[k] = c.P.G * pm.w * acc;
    }
    e[0] = f[0]; e[1] = f[1]; e[2] = f[2];
    e[3] = pm.y * f[2] - pm.z * f[1];
    e[4] = pm.z * f[0] - pm.x * f[2];
    e[5] = pm.x * f[1] - pm.y * f[0];
  }
}

struct SolveOut { bool converged; double best; bool assembled; double a_norm2; };

template <bool MIXED>
__device__ SolveOut newton_solve(const Ctx& c, double half, double* red, int* flag, int* iters, PhaseTimer& tm) {
  SolveOut o{false, kHuge, false, 0.0};
  load_world_state(c);  // vmid = current world velocity; snap = P_s^n
  __syncthreads();
  copy_bodies6(c, c.s.vm, c.s.best);
  __syncthreads();
  tm.lap(PH_OTHER);
  // The accepted line-search probe already evaluated PRE, the joint values and POST at the point
  // the next iteration starts from (newton.rs:383-395); only the Jacobian is missing there.
  bool carried = false;
  double carried_norm = 0.0;
  for (int it = 0; it < c.P.max_newton; ++it) {
    ++*iters;
    double rnorm;
    if (carried) {
      phase_joints<MIXED>(c, c.s.vm, true);
      __syncthreads();
      tm.lap(PH_JACOBIAN);
      rnorm = carried_norm;
      carried = false;
    } else {
      phase_pre(c, c.s.vm, half);
      __syncthreads();
      tm.lap(PH_PRE);
      phase_joints<MIXED>(c, c.s.vm, true);
      __syncthreads();
      tm.lap(PH_JACOBIAN);
      rnorm = phase_post(c, c.s.vm, half, red);
      copy_mass0(c);
    }
    if (rnorm < o.best) {
      o.best = rnorm;
      copy_bodies6(c, c.s.vm, c.s.best);
    }
    __syncthreads();
    tm.lap(PH_POST);
    if (rnorm <= c.P.tol2) { o.converged = true; break; }
    if (!(rnorm < kHuge)) break;
    o.a_norm2 = phase_assemble(c, half, red);
    o.assembled = true;
    tm.lap(PH_ASSEMBLE);
    phase_solve(c, flag);
    tm.lap(PH_SOLVE);
    // no correction at all -> hand over to sub-division (newton.rs:449-456)
    int nz = 0;
    for (int t = threadIdx.x; t < 6 * c.d.m; t += blockDim.x) nz |= (c.s.dv[t] != 0.0);
    if (!__syncthreads_or(nz)) break;
    copy_bodies6(c, c.s.vm, c.s.base);
    __syncthreads();
    int accepted = -1;
    double alpha = 1.0;
    for (int lane = 0; lane < 8; ++lane) {
      make_trial(c, alpha);
      __syncthreads();
      phase_pre(c, c.s.trial, half);
      __syncthreads();
      phase_joints<MIXED>(c, c.s.trial, false);
      __syncthreads();
      double tnorm = phase_post(c, c.s.trial, half, red);
      bool acc = tnorm < rnorm;
      if (lane == 0 || acc) copy_mass0(c);
      __syncthreads();
      if (acc) { accepted = lane; carried_norm = tnorm; break; }
      alpha = alpha / 2.0;
    }
    tm.lap(PH_LINE_SEARCH);
    if (accepted < 0) break;  // vm still holds the base iterate
    copy_bodies6(c, c.s.trial, c.s.vm);
    carried = true;  // mid, conn, mass, rhs and scale now describe the accepted iterate
    __syncthreads();
  }
  // restore the best iterate for the commit
  copy_bodies6(c, c.s.best, c.s.vm);
  __syncthreads();
  return o;
}

__device__ bool log2_floor(double v, int* e) {
  if (!(v > 0.0)) return false;
  double x = v;
  int k = 0;
  while (x >= 2.0) { x /= 2.0; ++k; if (k > 250) return false; }
  while (x < 1.0 && k > -250) { x *= 2.0; --k; }
  *e = k;
  return true;
}
__device__ int div_euclid(int a, int b) { int q = a / b; if (a % b < 0) q -= 1; return q; }

__device__ bool signal_log2(const Ctx& c, const SolveOut& o, double* red, int* r) {
  if (!o.assembled) return false;
  double s = 0.0;
  for (int t = threadIdx.x; t < 36 * c.d.m; t += blockDim.x) s += c.s.mass0[t] * c.s.mass0[t];
  double massn = block_sum(s, red);
  double stiff = ScalarTraits<double>::eff_zero(massn) ? 0.0 : o.a_norm2 / massn;
  return log2_floor(stiff, r);
}

// commit_span (newton.rs:708-753)
__device__ void commit_span(const Ctx& c, double span, double half, bool converged) {
  for (int i = threadIdx.x; i < c.d.m; i += blockDim.x) {
    int q = c.A.dn_body[c.d.dyn_off + i];
    int g = c.gbody(q);
    double m0[8], vb[6], e[8], pm[8], inv[8], vbody[6], v6[6], I9[9];
#pragma unroll
    for (int k = 0; k < 8; ++k) m0[k] = c.W.pose[(size_t)k * c.W.n + g];
#pragma unroll
    for (int k = 0; k < 9; ++k) I9[k] = c.W.inertia[(size_t)k * c.W.n + g];
    screw_from6(c.s.vm + 6 * q, vb);
    twist_exp(vb, half, e);
    motor_compose(m0, e, pm);
    motor_reverse(pm, inv);
    twist_transport(vb, inv, vbody);
    screw_to6(vbody, v6);
    double p6[6], pb[6], pw[6], psm[6];
    inertia_apply(I9, c.W.diagonal[g] != 0, false, c.W.mass[g], v6, p6);
    screw_from6(p6, pb);
    wrench_transport(pb, pm, pw);
    screw_to6(pw, psm);
    double pnew[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) pnew[k] = converged ? psm[k] * 2.0 - c.s.snap[6 * q + k] : psm[k];
    double en[8], mnew[8], minv[8], pnb[6], pbody[6], out6[6];
    twist_exp(vb, span, en);
    motor_compose(m0, en, mnew);
    motor_reverse(mnew, minv);
    screw_from6(pnew, pnb);
    wrench_transport(pnb, minv, pbody);
    screw_to6(pbody, out6);
#pragma unroll
    for (int k = 0; k < 8; ++k) c.W.pose[(size_t)k * c.W.n + g] = mnew[k];
#pragma unroll
    for (int k = 0; k < 6; ++k) c.W.mom[(size_t)k * c.W.n + g] = out6[k];
  }
}

template <bool MIXED>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_newton_step(NewtonDeviceArrays A, WorldRef W, const int* __restrict__ queue,
                                                         int n_islands, int* __restrict__ head) {
  __shared__ double red[kWarps];
  __shared__ int flag;
  __shared__ int item;
  __shared__ long long phase_acc[kPhases];
  if (threadIdx.x < kPhases) phase_acc[threadIdx.x] = 0;
  __syncthreads();
  PhaseTimer tm{phase_acc, 0};
  tm.start();
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(head, 1);
    __syncthreads();
    int k = item;
    __syncthreads();
    if (k >= n_islands) {
      if (threadIdx.x < kPhases) atomicAdd(reinterpret_cast<unsigned long long*>(&A.phase_cycles[threadIdx.x]),
                                           static_cast<unsigned long long>(phase_acc[threadIdx.x]));
      break;
    }
    Ctx c;
    c.A = A;
    c.island = queue[k];
    c.d = A.desc[c.island];
    if (!W.w_active[c.d.world]) continue;  // the world holds this step
    c.W = W;
    c.s = carve(A.scratch + c.d.scratch_off, c.d.nb, c.d.nj, c.d.m);
    {
      const exg_step_params_t& wp = W.wparams[c.d.world];
      c.P.dt = wp.dt;
      c.P.warp = wp.warp;
      c.P.tol2 = wp.tol * wp.tol;
      c.P.G = wp.G;
      c.P.max_newton = wp.max_newton > 0 ? wp.max_newton : 32;
      c.P.pose_factor_scale = (wp.newton_flags & EXG_NEWTON_EXACT_POSE_FACTOR) ? 0.5 : 1.0;
      c.P.splits = W.w_splits[c.d.world];
      c.P.nw = W.w_n[c.d.world];
      c.P.wbody_off = W.w_body_off[c.d.world];
      c.P.part = W.grav_partial + W.w_poff[c.d.world];
    }
    load_external(c);
    __syncthreads();
    unsigned long long remaining = 1ull << kMaxDepth;
    int depth = 0, spans = 0, iters = 0, maxdepth = 0;
    double last_best = 0.0;
    while (remaining > 0) {
      unsigned long long units = 1ull << (kMaxDepth - depth);
      while (units > remaining) { ++depth; units >>= 1; }
      double span = c.P.dt;
      for (int t = 0; t < depth; ++t) span = span / 2.0;
      double half = span / 2.0;
      ++spans;
      maxdepth = max(maxdepth, depth);
      SolveOut o = newton_solve<MIXED>(c, half, red, &flag, &iters, tm);
      last_best = o.best;
      bool finite = o.best < kHuge;
      bool last = depth == kMaxDepth;
      if (!o.converged && !last) {
        int r, down;
        if (signal_log2(c, o, red, &r)) down = div_euclid(r - kThresholdLog2, kPerHalvingLog2) + 1; else down = 1;
        depth += min(max(down, 1), kMaxDepth - depth);
        continue;
      }
      if (o.converged || finite) commit_span(c, span, half, o.converged);
      __syncthreads();
      tm.lap(PH_COMMIT);
      remaining -= units;
      auto aligned = [&](int dd) {
        if (dd <= 0) return false;
        unsigned long long bigger = 1ull << (kMaxDepth - (dd - 1));
        return bigger <= remaining && remaining % bigger == 0;
      };
      int r;
      if (remaining > 0 && o.converged && aligned(depth) && signal_log2(c, o, red, &r)) {
        int up = div_euclid(kThresholdLog2 - r, kPerHalvingLog2);
        while (up > 0 && aligned(depth)) { --depth; --up; }
      }
    }
    if (threadIdx.x == 0) {
      A.stats[4 * c.island + 0] = spans;
      A.stats[4 * c.island + 1] = iters;
      A.stats[4 * c.island + 2] = maxdepth;
      A.stats[4 * c.island + 3] = (last_best < kHuge) ? 0 : 1;
      A.residual[c.island] = last_best;
    }
    __syncthreads();
  }
}

}  // namespace

// ── host: island structure ────────────────────────────────────────────────────
long long newton_footprint_bytes(int nb, int nj) {
  // scratch, then the structure: 13 ints per body (body list, order, incidence pointers,
  // dynamic list, parents, levels, children, 3 assembly cells), 9 per joint plus its 10 params
  return ((scratch_doubles(nb, nj, nb) + 31) & ~31LL) * 8 + (long long)nb * 13 * 4 + (long long)nj * (9 * 4 + 80) +
         (long long)sizeof(IslandDesc) + 64;
}

NewtonWorld::~NewtonWorld() {
  d_desc.release();
  for (DevArr<int>* a : {&d_isl_body, &d_jl_law, &d_jl_a, &d_jl_b, &d_ib_order, &d_ib_inc_ptr, &d_ib_inc_ref, &d_dn_body,
                         &d_dn_parent, &d_lv_ptr, &d_lv_nodes, &d_ch_ptr, &d_ch_idx, &d_cell_ptr, &d_cell_terms, &d_stats,
                         &d_queue})
    a->release();
  d_jl_params.release();
  d_scratch.release();
  d_residual.release();
  d_phase.release();
}

int NewtonWorld::add_world(exg_device_s* dev, int slot, int body_off, const exg_body_t* bodies, int n,
                           const exg_joint_t* joints, int nj) {
  (void)dev;
  WorldSrc src;
  src.body_off = body_off;
  src.kin.resize(n);
  for (int i = 0; i < n; ++i) src.kin[i] = bodies[i].kinematic != 0;
  src.joints.assign(joints, joints + nj);
  int rc = build_world(slot, src);
  if (rc != EXG_OK) return rc;
  if ((int)src_.size() <= slot) src_.resize(slot + 1);
  src.live = true;
  src_[slot] = std::move(src);
  return EXG_OK;
}

// Rebuild the structure arrays from the live worlds alone, once removed worlds hold most of them.
void NewtonWorld::compact() {
  desc_.clear(); alive_.clear(); scratch_len_.clear();
  for (std::vector<int>* v : {&h_isl_body, &h_jl_law, &h_jl_a, &h_jl_b, &h_ib_order, &h_ib_inc_ptr, &h_ib_inc_ref,
                              &h_dn_body, &h_dn_parent, &h_lv_ptr, &h_lv_nodes, &h_ch_ptr, &h_ch_idx, &h_cell_ptr,
                              &h_cell_terms})
    v->clear();
  h_jl_params.clear();
  world_islands_.clear();
  scratch_alloc_.init(scratch_alloc_.capacity());
  n_live_ = 0;
  for (int slot = 0; slot < (int)src_.size(); ++slot)
    if (src_[slot].live) build_world(slot, src_[slot]);  // rebuilt worlds were accepted before
  d_desc.size = 0;
  for (DevArr<int>* a : {&d_isl_body, &d_jl_law, &d_jl_a, &d_jl_b, &d_ib_order, &d_ib_inc_ptr, &d_ib_inc_ref, &d_dn_body,
                         &d_dn_parent, &d_lv_ptr, &d_lv_nodes, &d_ch_ptr, &d_ch_idx, &d_cell_ptr, &d_cell_terms})
    a->size = 0;
  d_jl_params.size = 0;
  dirty_ = true;
}

int NewtonWorld::build_world(int slot, const WorldSrc& src) {
  const int n = (int)src.kin.size(), nj = (int)src.joints.size(), body_off = src.body_off;
  const exg_joint_t* joints = src.joints.data();
  // islands = connected components of the world's joint graph, bodies ascending, joints ascending
  std::vector<int> parent(n);
  for (int i = 0; i < n; ++i) parent[i] = i;
  std::function<int(int)> find = [&](int x) {
    while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
    return x;
  };
  for (int k = 0; k < nj; ++k) {
    int ra = find(joints[k].a), rb = find(joints[k].b);
    if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
  }
  std::vector<int> isl_of_root(n, -1);
  std::vector<std::vector<int>> ib, ij;
  for (int i = 0; i < n; ++i) {
    int r = find(i);
    if (isl_of_root[r] < 0) { isl_of_root[r] = (int)ib.size(); ib.emplace_back(); ij.emplace_back(); }
    ib[isl_of_root[r]].push_back(i);
  }
  for (int k = 0; k < nj; ++k) ij[isl_of_root[find(joints[k].a)]].push_back(k);

  // build into staging vectors first, so a refused world leaves the structure untouched
  std::vector<IslandDesc> desc;
  std::vector<long long> lens;
  std::vector<int> s_isl_body, s_jl_law, s_jl_a, s_jl_b, s_ib_order, s_ib_inc_ptr, s_ib_inc_ref, s_dn_body, s_dn_parent,
      s_lv_ptr, s_lv_nodes, s_ch_ptr, s_ch_idx, s_cell_ptr, s_cell_terms;
  std::vector<double> s_jl_params;
  const int base_isl_body = (int)h_isl_body.size(), base_jl = (int)h_jl_law.size(), base_order = (int)h_ib_order.size(),
            base_inc_ptr = (int)h_ib_inc_ptr.size(), base_inc_ref = (int)h_ib_inc_ref.size(),
            base_dn = (int)h_dn_body.size(), base_lv = (int)h_lv_ptr.size(), base_ch_idx = (int)h_ch_idx.size(),
            base_cell_ptr = (int)h_cell_ptr.size(), base_cell_terms = (int)h_cell_terms.size();
  std::vector<int> local(n, -1);
  for (size_t I = 0; I < ib.size(); ++I) {
    const std::vector<int>& B = ib[I];
    const std::vector<int>& J = ij[I];
    IslandDesc d;
    d.world = slot;
    d.body_off = base_isl_body + (int)s_isl_body.size();
    d.nb = (int)B.size();
    d.joint_off = base_jl + (int)s_jl_law.size();
    d.nj = (int)J.size();
    const int jl0 = (int)s_jl_law.size();
    for (int q = 0; q < d.nb; ++q) { local[B[q]] = q; s_isl_body.push_back(body_off + B[q]); }
    for (int q = 0; q < d.nj; ++q) {
      const exg_joint_t& jt = joints[J[q]];
      s_jl_law.push_back(jt.law);
      s_jl_a.push_back(local[jt.a]);
      s_jl_b.push_back(local[jt.b]);
      for (int k = 0; k < 10; ++k) s_jl_params.push_back(jt.params[k]);
    }
    // dynamic order (island order, kinematic excluded)
    std::vector<int> order(d.nb, -1), dyn_body;
    for (int q = 0; q < d.nb; ++q)
      if (!src.kin[B[q]]) { order[q] = (int)dyn_body.size(); dyn_body.push_back(q); }
    const int m = (int)dyn_body.size();
    d.m = m;
    d.dyn_off = base_dn + (int)s_dn_body.size();
    for (int q = 0; q < d.nb; ++q) s_ib_order.push_back(order[q]);
    // incidence per island body in joint order (the reference's gather order)
    d.inc_off = base_inc_ptr + (int)s_ib_inc_ptr.size();
    {
      std::vector<std::vector<int>> inc(d.nb);
      for (int q = 0; q < d.nj; ++q) {
        inc[s_jl_a[jl0 + q]].push_back(2 * q);
        inc[s_jl_b[jl0 + q]].push_back(2 * q + 1);
      }
      int pos = base_inc_ref + (int)s_ib_inc_ref.size();
      for (int q = 0; q < d.nb; ++q) {
        s_ib_inc_ptr.push_back(pos);
        for (int r : inc[q]) { s_ib_inc_ref.push_back(r); ++pos; }
      }
      s_ib_inc_ptr.push_back(pos);
    }
    // dynamic adjacency (distinct neighbours)
    std::vector<std::vector<int>> adj(m);
    for (int q = 0; q < d.nj; ++q) {
      int ea = order[s_jl_a[jl0 + q]], eb = order[s_jl_b[jl0 + q]];
      if (ea < 0 || eb < 0) continue;
      if (std::find(adj[ea].begin(), adj[ea].end(), eb) == adj[ea].end()) adj[ea].push_back(eb);
      if (std::find(adj[eb].begin(), adj[eb].end(), ea) == adj[eb].end()) adj[eb].push_back(ea);
    }
    // forest check; elimination tree rooted at each component's centre
    std::vector<int> par(m, -2), level(m, 0), comp_of(m, -1), dist(m, -1), du(m, -1), dc(m, -1);
    long edges = 0;
    for (int i = 0; i < m; ++i) edges += (long)adj[i].size();
    edges /= 2;
    int comps = 0;
    auto bfs = [&](int root, std::vector<int>& dd, std::vector<int>& seen) {
      seen.clear();
      seen.push_back(root);
      dd[root] = 0;
      for (size_t h = 0; h < seen.size(); ++h)
        for (int nb2 : adj[seen[h]])
          if (dd[nb2] < 0) { dd[nb2] = dd[seen[h]] + 1; seen.push_back(nb2); }
    };
    std::vector<int> seen, seen_u, seen_c;
    for (int st = 0; st < m; ++st) {
      if (comp_of[st] >= 0) continue;
      bfs(st, dist, seen);
      for (int x : seen) comp_of[x] = comps;
      int u = seen.back();
      bfs(u, du, seen_u);
      int v = seen_u.back();
      std::vector<int> path{v};
      while (path.back() != u) {
        int cur = path.back();
        for (int nb2 : adj[cur]) if (du[nb2] == du[cur] - 1) { path.push_back(nb2); break; }
      }
      int centre = path[path.size() / 2];
      bfs(centre, dc, seen_c);
      par[centre] = -1;
      for (int x : seen_c) {
        level[x] = dc[x];
        for (int nb2 : adj[x]) if (dc[nb2] == dc[x] + 1 && par[nb2] == -2) par[nb2] = x;
      }
      ++comps;
    }
    for (int q = 0; q < d.nb; ++q) local[B[q]] = -1;
    if (edges != m - comps) return EXG_ERR_UNSUPPORTED;  // a cycle among the dynamic bodies
    int nlev = 0;
    for (int i = 0; i < m; ++i) nlev = std::max(nlev, level[i] + 1);
    d.n_levels = nlev;
    d.lv_off = base_lv + (int)s_lv_ptr.size();
    {
      std::vector<std::vector<int>> by(nlev);
      for (int i = 0; i < m; ++i) by[level[i]].push_back(i);
      int acc = 0;
      for (int L = 0; L < nlev; ++L) {
        s_lv_ptr.push_back(acc);
        for (int i : by[L]) s_lv_nodes.push_back(i);
        acc += (int)by[L].size();
      }
      s_lv_ptr.push_back(acc);
    }
    // children: one absolute offset into ch_idx per node (a sentinel follows the last node of
    // all islands), island-relative node indices in ch_idx
    {
      std::vector<std::vector<int>> ch(m);
      for (int i = 0; i < m; ++i) if (par[i] >= 0) ch[par[i]].push_back(i);
      for (int i = 0; i < m; ++i) {
        s_ch_ptr.push_back(base_ch_idx + (int)s_ch_idx.size());
        for (int x : ch[i]) s_ch_idx.push_back(x);
      }
      for (int i = 0; i < m; ++i) { s_dn_body.push_back(dyn_body[i]); s_dn_parent.push_back(par[i]); }
    }
    // assembly cells: (node, kind) with kind 0 = diagonal, 1 = (node row, parent col),
    // 2 = (parent row, node col)
    d.cell_off = base_cell_ptr + (int)s_cell_ptr.size();
    {
      std::vector<std::vector<int>> cells(3 * m);
      for (int q = 0; q < d.nj; ++q) {
        int ends[2] = {order[s_jl_a[jl0 + q]], order[s_jl_b[jl0 + q]]};
        for (int re = 0; re < 2; ++re) {
          if (ends[re] < 0) continue;
          for (int ce = 0; ce < 2; ++ce) {
            if (ends[ce] < 0) continue;
            int row = ends[re], col = ends[ce], target;
            if (row == col) target = 3 * row + 0;
            else if (par[row] == col) target = 3 * row + 1;
            else if (par[col] == row) target = 3 * col + 2;
            else return EXG_ERR_UNSUPPORTED;
            cells[target].push_back(q * 4 + re * 2 + ce);
          }
        }
      }
      int pos = base_cell_terms + (int)s_cell_terms.size();
      for (int t = 0; t < 3 * m; ++t) {
        s_cell_ptr.push_back(pos);
        for (int x : cells[t]) { s_cell_terms.push_back(x); ++pos; }
      }
      s_cell_ptr.push_back(pos);
    }
    desc.push_back(d);
    lens.push_back((scratch_doubles(d.nb, d.nj, m) + 31) & ~31LL);
  }
  // scratch ranges (grow the scratch array when the allocator has no room)
  for (size_t I = 0; I < desc.size(); ++I) {
    long long off = scratch_alloc_.alloc(lens[I]);
    if (off < 0) {
      long long old = scratch_alloc_.capacity();
      long long grow = std::max(old, lens[I] + 1024);
      scratch_alloc_.grow(old + grow);
      off = scratch_alloc_.alloc(lens[I]);
    }
    desc[I].scratch_off = off;
  }
  // commit the staging vectors
  auto cat = [](std::vector<int>& dst, const std::vector<int>& src) { dst.insert(dst.end(), src.begin(), src.end()); };
  cat(h_isl_body, s_isl_body); cat(h_jl_law, s_jl_law); cat(h_jl_a, s_jl_a); cat(h_jl_b, s_jl_b);
  cat(h_ib_order, s_ib_order); cat(h_ib_inc_ptr, s_ib_inc_ptr); cat(h_ib_inc_ref, s_ib_inc_ref);
  cat(h_dn_body, s_dn_body); cat(h_dn_parent, s_dn_parent); cat(h_lv_ptr, s_lv_ptr); cat(h_lv_nodes, s_lv_nodes);
  cat(h_ch_ptr, s_ch_ptr); cat(h_ch_idx, s_ch_idx); cat(h_cell_ptr, s_cell_ptr); cat(h_cell_terms, s_cell_terms);
  h_jl_params.insert(h_jl_params.end(), s_jl_params.begin(), s_jl_params.end());
  if ((int)world_islands_.size() <= slot) world_islands_.resize(slot + 1);
  world_islands_[slot].clear();
  for (size_t I = 0; I < desc.size(); ++I) {
    world_islands_[slot].push_back((int)desc_.size());
    desc_.push_back(desc[I]);
    alive_.push_back(1);
    scratch_len_.push_back(lens[I]);
    ++n_live_;
  }
  dirty_ = true;
  return EXG_OK;
}

void NewtonWorld::remove_world(int slot) {
  if (slot < 0 || slot >= (int)world_islands_.size()) return;
  for (int I : world_islands_[slot]) {
    if (!alive_[I]) continue;
    alive_[I] = 0;
    scratch_alloc_.release(desc_[I].scratch_off, scratch_len_[I]);
    --n_live_;
  }
  world_islands_[slot].clear();
  if (slot < (int)src_.size()) src_[slot] = WorldSrc();
  dirty_ = true;
}

int NewtonWorld::sync(exg_device_s* dev, cudaStream_t s) {
  (void)dev;
  if (!dirty_) return EXG_OK;
  if ((long long)desc_.size() > 1024 && (long long)desc_.size() > 2LL * n_live_) compact();
  int rc = EXG_OK;
  auto up = [&](auto& d, const auto& h) {
    if (rc == EXG_OK && (long long)h.size() > d.size) rc = d.append(h.data() + d.size, (long long)h.size() - d.size, s);
  };
  up(d_desc, desc_);
  up(d_isl_body, h_isl_body); up(d_jl_law, h_jl_law); up(d_jl_a, h_jl_a); up(d_jl_b, h_jl_b);
  up(d_jl_params, h_jl_params); up(d_ib_order, h_ib_order); up(d_ib_inc_ptr, h_ib_inc_ptr);
  up(d_ib_inc_ref, h_ib_inc_ref); up(d_dn_body, h_dn_body); up(d_dn_parent, h_dn_parent); up(d_lv_ptr, h_lv_ptr);
  up(d_lv_nodes, h_lv_nodes); up(d_ch_idx, h_ch_idx); up(d_cell_ptr, h_cell_ptr); up(d_cell_terms, h_cell_terms);
  if (rc != EXG_OK) return rc;
  // ch_ptr carries a sentinel after its last entry; rewrite it with the tail
  if ((long long)h_ch_ptr.size() > d_ch_ptr.size || d_ch_ptr.cap == 0) {
    long long from = d_ch_ptr.size;
    std::vector<int> tail(h_ch_ptr.begin() + from, h_ch_ptr.end());
    tail.push_back((int)h_ch_idx.size());
    rc = d_ch_ptr.append(tail.data(), (long long)tail.size(), s);
    if (rc != EXG_OK) return rc;
    d_ch_ptr.size -= 1;  // the sentinel is overwritten by the next append
  }
  // scratch: per-step contents only, so growth needs no copy
  if (d_scratch.cap < scratch_alloc_.capacity()) {
    d_scratch.release();
    rc = d_scratch.reserve(std::max<long long>(scratch_alloc_.capacity(), 1), s);
    if (rc != EXG_OK) return rc;
  }
  long long ni = (long long)desc_.size();
  if ((rc = d_stats.reserve(std::max<long long>(4 * ni, 4), s)) != EXG_OK) return rc;
  if ((rc = d_residual.reserve(std::max<long long>(ni, 1), s)) != EXG_OK) return rc;
  if (d_phase.cap == 0) {
    std::vector<long long> z(kPhases, 0);
    if ((rc = d_phase.assign(z.data(), kPhases, s)) != EXG_OK) return rc;
  }
  // queue of live islands, largest first, then the scheduler's counter
  std::vector<int> q;
  for (int I = 0; I < (int)desc_.size(); ++I) if (alive_[I]) q.push_back(I);
  std::stable_sort(q.begin(), q.end(),
                   [&](int a, int b) { return desc_[a].nb + desc_[a].nj > desc_[b].nb + desc_[b].nj; });
  q.push_back(0);
  if ((rc = d_queue.assign(q.data(), (long long)q.size(), s)) != EXG_OK) return rc;
  arr = NewtonDeviceArrays{d_desc.ptr,      d_isl_body.ptr, d_jl_law.ptr,   d_jl_a.ptr,      d_jl_b.ptr,     d_jl_params.ptr,
                           d_ib_order.ptr,  d_ib_inc_ptr.ptr, d_ib_inc_ref.ptr, d_dn_body.ptr, d_dn_parent.ptr, d_lv_ptr.ptr,
                           d_lv_nodes.ptr,  d_ch_ptr.ptr,   d_ch_idx.ptr,   d_cell_ptr.ptr,  d_cell_terms.ptr, d_scratch.ptr,
                           d_stats.ptr,     d_residual.ptr, d_phase.ptr};
  dirty_ = false;
  return EXG_OK;
}

int NewtonWorld::enqueue(exg_device_s* dev, DeviceWorld& w, cudaStream_t s) {
  if (n_live_ == 0) return EXG_OK;
  if (dirty_) return EXG_ERR_INVALID_ARGUMENT;  // sync() first
  WorldRef W{w.pose,    w.mom,    w.mass,   w.inertia, w.kinematic,  w.diagonal, w.pos_mass,
             w.grav_partial, w.wparams, w.w_poff, w.w_splits, w.w_n, w.w_body_off, w.w_active, w.n};
  int* head = d_queue.ptr + n_live_;
  // persistent CTAs: as many as can be resident at once
  static int resident[2] = {0, 0};
  const int mixed = w.precision == EXG_PRECISION_MIXED;
  if (resident[mixed] == 0) {
    int per_sm = 0;
    cudaError_t e = mixed ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_newton_step<true>, kThreads, 0)
                          : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_newton_step<false>, kThreads, 0);
    resident[mixed] = (e == cudaSuccess && per_sm > 0) ? per_sm : 1;
  }
  int grid = std::min(n_live_, std::max(1, dev->sm_count) * resident[mixed]);
  EXG_CUDA_TRY(cudaMemsetAsync(head, 0, sizeof(int), s));
  int tok = prof_begin(dev, PROF_NEWTON, s);
  if (mixed)
    k_newton_step<true><<<grid, kThreads, 0, s>>>(arr, W, d_queue.ptr, n_live_, head);
  else
    k_newton_step<false><<<grid, kThreads, 0, s>>>(arr, W, d_queue.ptr, n_live_, head);
  prof_end(dev, tok, s);
  return exg_after_launch(dev);
}

int NewtonWorld::read_phase_cycles(long long* out) {
  for (int k = 0; k < kPhases; ++k) out[k] = 0;
  if (d_phase.cap == 0) return EXG_OK;
  EXG_CUDA_TRY(cudaMemcpy(out, d_phase.ptr, sizeof(long long) * kPhases, cudaMemcpyDeviceToHost));
  return EXG_OK;
}

int NewtonWorld::read_stats(int world, exg_world_stats_t* st) {
  const int ni = (int)desc_.size();
  std::vector<int> stats(4 * (size_t)std::max(ni, 1));
  std::vector<double> res(std::max(ni, 1));
  if (ni > 0 && d_stats.cap >= 4LL * ni) {
    EXG_CUDA_TRY(cudaMemcpy(stats.data(), d_stats.ptr, sizeof(int) * 4 * ni, cudaMemcpyDeviceToHost));
    EXG_CUDA_TRY(cudaMemcpy(res.data(), d_residual.ptr, sizeof(double) * ni, cudaMemcpyDeviceToHost));
  }
  int spans = 0, iters = 0, depth = 0, fatal = 0;
  double worst = 0.0;
  for (int I = 0; I < ni; ++I) {
    if (!alive_[I]) continue;
    if (world >= 0 && desc_[I].world != world) continue;
    spans = std::max(spans, stats[4 * I]);
    iters = std::max(iters, stats[4 * I + 1]);
    depth = std::max(depth, stats[4 * I + 2]);
    fatal |= stats[4 * I + 3];
    worst = std::max(worst, res[I]);
  }
  st->last_spans = spans;
  st->last_newton_iterations = iters;
  st->max_depth_reached = depth;
  st->fatal = fatal;
  st->last_residual = worst;
  return EXG_OK;
}

// ── host energy (the same algebra compiled for the host) ──────────────────────
double host_world_energy(const exg_body_t* b, int n, const exg_joint_t* joints, int nj, const exg_step_params_t& p) {
  double e = 0.0;
  std::vector<double> pos(3 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    exg::body_position(b[i].pose, &pos[3 * i]);
    if (b[i].kinematic) continue;
    double v6[6];
    exg::inertia_inverse(b[i].inertia, b[i].diagonal != 0, false, b[i].mass, b[i].momentum, v6);
    double mb[6], vb[6];
    exg::screw_from6(b[i].momentum, mb);
    exg::screw_from6(v6, vb);
    e += 0.5 * exg::screw_power(mb, vb);
  }
  if (p.gravity_law != EXG_GRAVITY_OFF) {
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) {
        if (b[i].kinematic || b[j].kinematic) continue;
        double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1], dz = pos[3 * j + 2] - pos[3 * i + 2];
        double r2 = dx * dx + dy * dy + dz * dz, mm = p.G * b[i].mass * b[j].mass;
        if (p.gravity_law == EXG_GRAVITY_PLUMMER) e -= mm / std::sqrt(r2 + p.softening * p.softening);
        else {
          double d = std::sqrt(r2), sz = b[j].size;
          e -= d >= sz ? mm / d : mm * (3.0 * sz * sz - r2) / (2.0 * sz * sz * sz);
        }
      }
  }
  for (int k = 0; k < nj; ++k) {
    const exg_joint_t& j = joints[k];
    if (j.law > 1) continue;
    double pa[4], pb[4], line[6];
    exg::anchor_point(b[j.a].pose, j.params, pa);
    exg::anchor_point(b[j.b].pose, j.params + 3, pb);
    exg::point_join(pa, pb, line);
    double d = exg::soft_weight_norm(line, j.params[9]);
    double dl = d - j.params[6];
    e += 0.5 * j.params[7] * dl * dl;
  }
  return e;
}
