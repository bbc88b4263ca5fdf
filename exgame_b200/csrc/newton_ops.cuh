// Per-item operations of the device Newton step, shared by the two schedules that run it:
//   the island kernel (one CTA per island, newton.cu) and
//   the wave schedule (every phase a grid-wide kernel over all large islands, newton_wave.cu).
// Each operation works on one body, joint task, dynamic node or assembly cell of one island, so
// both schedules do the same arithmetic in the same order for every item; only the order in
// which items run differs, and no result depends on it.
#pragma once
#include "body.cuh"
#include "joint_eval.cuh"
#include "world_newton.cuh"

namespace exg_newton {

using namespace exg;

constexpr int kMaxDepth = 8;        // solve_step budget: MAX_DEPTH (newton.rs:63-74)
constexpr int kThresholdLog2 = 8;   // THRESHOLD_LOG2
constexpr int kPerHalvingLog2 = 4;  // PER_HALVING_LOG2
constexpr double kHuge = 1e9;
constexpr double kFloor2 = 1e-9 * 1e-9;
constexpr int kJacStride = 36;  // per (joint, slice): d[36] (144 B in FP32, 16-byte aligned records)
constexpr int kLineSearchLanes = 8;
// Assembly terms carry this bit when the joint's law is the torsional damper, whose Jacobian
// slices are known in closed form (joint_jacobian_part): the wave reads no slices for them.
constexpr int kTermTorsional = 1 << 30;

struct Scratch {
  double *vm, *base, *best, *trial, *mid, *snap, *ext, *conn, *jac, *mass, *mass0, *rhs, *scale, *D, *Dinv, *Acp, *Apc, *S,
      *bvec, *dv, *G;
};

// Doubles of an island's scratch; n_slots (block-LU islands) adds the off-diagonal block pairs.
EXG_HD long long scratch_doubles(int nb, int nj, int m, int n_slots = 0) {
  return (long long)nb * (6 * 4 + 8 + 6 * 2) + (long long)nj * (6 + 4 * kJacStride) + (long long)m * (36 * 7 + 6 * 3 + 2) +
         (long long)n_slots * 72;
}

// The island's scratch arrays; a block-LU island's off-diagonal blocks (G) follow the common ones,
// so a tree island's layout does not depend on the solver.
__device__ inline Scratch carve(double* p, int nb, int nj, int m, int n_slots = 0) {
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
  s.G = p; p += (size_t)n_slots * 72;
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

// The island's world parameters.
struct IslandParams {
  double dt, warp, tol2, G, pose_factor_scale;
  int max_newton;
  bool ns_pivot;  // Newton-Schulz pivot inverses (mixed path, EXG_NEWTON_NS_PIVOT)
  int splits, nw, wbody_off;
  const double* part;
};

// An island's frame for one step: its poses are read relative to an anchor near the island's centre
// of mass at the step's start, and written back to world coordinates. The reference keeps each
// island's poses local to an origin re-bound to its centre of mass after every step
// (Island::recompute_centroid, crates/newton/src/mechanism/island.rs:206-243;
// crates/newton/tests/precision_seam.rs measures why): world-origin twists (v = v_body - w x p)
// cancel catastrophically far from the origin. Here the anchor is the centre of mass rounded to a
// multiple of kFrameGrid in each component, so an island within kFrameGrid / 2 of the origin steps
// in world coordinates exactly as before: the Newton residual's per-body angular scale
// (functions/src/lib.rs:170-247) is taken about the frame's origin and has a floor of 1e-9, which a
// small island's bodies at its own centre of mass reach, and a 1e-10 tolerance then cannot be met.
// Layout (doubles): [0, 3) the anchor a, [4, 12) the translator by -a, [12, 20) the one by +a.
constexpr double kFrameGrid = 1024.0;
constexpr int kFrameDoubles = 20;
__device__ inline void frame_make(const double* a, double* f) {
  double t6[6] = {-a[0], -a[1], -a[2], 0.0, 0.0, 0.0}, b[6];
  f[0] = a[0]; f[1] = a[1]; f[2] = a[2]; f[3] = 0.0;
  screw_from6(t6, b);
  twist_exp(b, 1.0, f + 4);
  t6[0] = a[0]; t6[1] = a[1]; t6[2] = a[2];
  screw_from6(t6, b);
  twist_exp(b, 1.0, f + 12);
}

// The frame of island d for this step, by a CTA of kFrameThreads threads (the wave and the island
// kernel both call this, so both get the same bits): thread t sums m p over the island's bodies
// t, t + kFrameThreads, ... in island order (kinematic bodies weigh nothing), then a fixed tree over
// the threads; the centre of mass is the sum over the mass (the island's first body where the
// island has no dynamic mass), and the anchor that point on the kFrameGrid grid. sh:
// 4 * kFrameThreads doubles of shared memory; f receives the frame.
constexpr int kFrameThreads = 256;
__device__ inline void island_frame(const NewtonDeviceArrays& A, const WorldRef& W, const IslandDesc& d, double* sh,
                                    double* f) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int q = threadIdx.x; q < d.nb; q += kFrameThreads) {
    const int g = A.isl_body[d.body_off + q];
    const double m = W.kinematic[g] ? 0.0 : W.mass[g];
    double pose[8], p3[3];
#pragma unroll
    for (int e = 0; e < 8; ++e) pose[e] = W.pose[(size_t)e * W.n + g];
    body_position(pose, p3);
    acc[0] += p3[0] * m;
    acc[1] += p3[1] * m;
    acc[2] += p3[2] * m;
    acc[3] += m;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) sh[4 * threadIdx.x + k] = acc[k];
  __syncthreads();
  for (int h = kFrameThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
#pragma unroll
      for (int k = 0; k < 4; ++k) sh[4 * threadIdx.x + k] += sh[4 * (threadIdx.x + h) + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double a[3];
    if (sh[3] > 0.0) {
      const double inv = 1.0 / sh[3];
      a[0] = sh[0] * inv; a[1] = sh[1] * inv; a[2] = sh[2] * inv;
    } else {
      const int g = A.isl_body[d.body_off];
      double pose[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) pose[e] = W.pose[(size_t)e * W.n + g];
      body_position(pose, a);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) a[k] = kFrameGrid * rint(a[k] / kFrameGrid);
    frame_make(a, f);
  }
  __syncthreads();
}

struct Ctx {
  NewtonDeviceArrays A;
  IslandDesc d;
  WorldRef W;
  IslandParams P;
  Scratch s;
  const double* frame;  // kFrameDoubles: the island's frame for this step (see frame_make)
  int island;
  EXG_HD int gbody(int q) const { return A.isl_body[d.body_off + q]; }
};

__device__ inline void resolve_params(Ctx& c) {
  const exg_step_params_t& wp = c.W.wparams[c.d.world];
  c.P.dt = wp.dt;
  c.P.warp = wp.warp;
  c.P.tol2 = wp.tol * wp.tol;
  c.P.G = wp.G;
  c.P.max_newton = wp.max_newton > 0 ? wp.max_newton : 32;
  c.P.pose_factor_scale = (wp.newton_flags & EXG_NEWTON_EXACT_POSE_FACTOR) ? 0.5 : 1.0;
  c.P.ns_pivot = (wp.newton_flags & EXG_NEWTON_NS_PIVOT) != 0;
  c.P.splits = c.W.w_splits[c.d.world];
  c.P.nw = c.W.w_n[c.d.world];
  c.P.wbody_off = c.W.w_body_off[c.d.world];
  c.P.part = c.W.grav_partial + c.W.w_poff[c.d.world];
}

__device__ inline Ctx make_ctx(const NewtonDeviceArrays& A, const WorldRef& W, int island) {
  Ctx c;
  c.A = A;
  c.W = W;
  c.island = island;
  c.d = A.desc[island];
  c.s = carve(A.scratch + c.d.scratch_off, c.d.nb, c.d.nj, c.d.m, c.d.n_slots);
  c.frame = nullptr;
  resolve_params(c);
  return c;
}

// A context from a descriptor the caller already holds (the wave keeps a copy per wave slot);
// c.island is then not set. `params` resolves the world's step parameters.
__device__ __forceinline__ Ctx make_ctx_desc(const NewtonDeviceArrays& A, const WorldRef& W, const IslandDesc& d,
                                             bool params) {
  Ctx c;
  c.A = A;
  c.W = W;
  c.island = -1;
  c.d = d;
  c.s = carve(A.scratch + c.d.scratch_off, c.d.nb, c.d.nj, c.d.m, c.d.n_slots);
  c.frame = nullptr;
  if (params) resolve_params(c);
  return c;
}

// The island's structure and scratch only (for operations that read no world parameter).
__device__ inline Ctx make_ctx_lite(const NewtonDeviceArrays& A, const WorldRef& W, int island) {
  Ctx c;
  c.A = A;
  c.W = W;
  c.island = island;
  c.d = A.desc[island];
  c.s = carve(A.scratch + c.d.scratch_off, c.d.nb, c.d.nj, c.d.m, c.d.n_slots);
  c.frame = nullptr;
  return c;
}

__device__ inline double nan_max(double a, double b) {
  if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000ULL);
  return a > b ? a : b;
}

// N doubles (N even) between registers and 16-byte aligned memory, two at a time (every scratch
// array starts on a 16-byte boundary and holds its items at even offsets).
template <int N>
__device__ __forceinline__ void ld_n(const double* p, double* o) {
  const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int e = 0; e < N / 2; ++e) { const double2 x = q[e]; o[2 * e] = x.x; o[2 * e + 1] = x.y; }
}
template <int N>
__device__ __forceinline__ void st_n(double* p, const double* v) {
  double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int e = 0; e < N / 2; ++e) q[e] = make_double2(v[2 * e], v[2 * e + 1]);
}

// ── per-item operations ─────────────────────────────────────────────────────
// PRE (functions::pre): mid = exp(half/2 x) * pose of island body q.
// Pose of world body g in the island's frame.
__device__ __forceinline__ void local_pose(const Ctx& c, int g, double* pose) {
  double w[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) w[k] = c.W.pose[(size_t)k * c.W.n + g];
  motor_compose(w, c.frame + 4, pose);
}

__device__ inline void op_pre(const Ctx& c, const double* x, double half, int q) {
  int g = c.gbody(q);
  double pose[8], xv[6], vb[6], e[8], m[8];
  local_pose(c, g, pose);
  ld_n<6>(x + 6 * (size_t)q, xv);
  screw_from6(xv, vb);
  twist_exp(vb, half, e);
  motor_compose(pose, e, m);
  st_n<8>(c.s.mid + 8 * (size_t)q, m);
}

// Jacobian slice storage: FP32 in the mixed path (the slices are FP32 duals, so nothing is lost),
// FP64 otherwise. Slice s of joint q: its 6x6 derivative block d[36] (row-major) at (q * 4 + s) *
// kJacStride. The slices' value parts are not stored: the residual takes the FP64 values (conn).
template <bool MIXED> struct JacType { typedef double T; };
template <> struct JacType<true> { typedef float T; };
template <bool MIXED>
__device__ inline typename JacType<MIXED>::T* jac_slice(const Ctx& c, int q, int slice) {
  return reinterpret_cast<typename JacType<MIXED>::T*>(c.s.jac) + ((size_t)q * 4 + slice) * kJacStride;
}

// The FP64 value of joint q at (mid, x): conn[q] = the wrench on end a. LAW >= 0 promises the
// joint's law at compile time (the other laws' code then drops out of the caller).
template <int LAW = -1>
__device__ inline void op_joint_value(const Ctx& c, const double* x, int q) {
  const int joff = c.d.joint_off;
  const int a = c.A.jl_a[joff + q], b = c.A.jl_b[joff + q];
  double ma[8], mb[8], xa[6], xb[6], out[12];
  ld_n<8>(c.s.mid + 8 * (size_t)a, ma);
  ld_n<8>(c.s.mid + 8 * (size_t)b, mb);
  ld_n<6>(x + 6 * (size_t)a, xa);
  ld_n<6>(x + 6 * (size_t)b, xb);
  joint_plain<double>(LAW >= 0 ? LAW : c.A.jl_law[joff + q], c.A.jl_params + 10 * (size_t)(joff + q), ma, mb, xa, xb,
                      c.P.dt, c.P.warp, out);
  st_n<6>(c.s.conn + 6 * (size_t)q, out);
}

// Jacobian slice `slice` of joint q at (mid, x). MIXED evaluates the derivative slices in FP32
// duals; the values that enter the residual always come from an FP64 evaluation (op_joint_value,
// or in FP64 the dual's value part, which equals it bit for bit: write_conn on slice 0), so the
// converged iterate is an FP64 solution whatever the Jacobian's precision.
// Half of slice `slice` (axes 6 slice + 3 half .. + 2) of joint q at (mid, x), into the slice's
// record at dst: its three derivative columns. Two halves make the slice bit for bit
// (joint_jacobian_part).
template <bool MIXED, int LAW = -1, int KIND = -1>
__device__ inline void op_joint_half_slice(const Ctx& c, const double* x, int q, int slice, int half, bool write_conn,
                                           typename JacType<MIXED>::T* dst) {
  typedef typename JacType<MIXED>::T J;
  const int joff = c.d.joint_off;
  const int a = c.A.jl_a[joff + q], b = c.A.jl_b[joff + q];
  const int law = LAW >= 0 ? LAW : c.A.jl_law[joff + q];
  const double* prm = c.A.jl_params + 10 * (size_t)(joff + q);
  J pa[8], pb[8], va[6], vb[6], val[6];
  {
    double ma[8], mb[8], xa[6], xb[6];
    ld_n<8>(c.s.mid + 8 * (size_t)a, ma);
    ld_n<8>(c.s.mid + 8 * (size_t)b, mb);
    ld_n<6>(x + 6 * (size_t)a, xa);
    ld_n<6>(x + 6 * (size_t)b, xb);
#pragma unroll
    for (int k = 0; k < 8; ++k) { pa[k] = J(ma[k]); pb[k] = J(mb[k]); }
#pragma unroll
    for (int k = 0; k < 6; ++k) { va[k] = J(xa[k]); vb[k] = J(xb[k]); }
  }
  joint_jacobian_part<J, 3, KIND>(law, prm, pa, pb, va, vb, c.P.dt, c.P.warp, slice, half, val, dst);
  if (!MIXED && write_conn && slice == 0 && half == 0) {
#pragma unroll
    for (int r = 0; r < 6; ++r) c.s.conn[6 * q + r] = double(val[r]);
  }
}

// The slice's 36 derivatives go to `dst` when given (a staging buffer), else to the island's scratch.
template <bool MIXED, int LAW = -1>
__device__ inline void op_joint_slice(const Ctx& c, const double* x, int q, int slice, bool write_conn,
                                      typename JacType<MIXED>::T* dst = nullptr) {
  const int joff = c.d.joint_off;
  const int a = c.A.jl_a[joff + q], b = c.A.jl_b[joff + q];
  const int law = LAW >= 0 ? LAW : c.A.jl_law[joff + q];
  const double* prm = c.A.jl_params + 10 * (size_t)(joff + q);
  if (MIXED) {
    float* o = dst ? reinterpret_cast<float*>(dst) : jac_slice<true>(c, q, slice);
    float pa[8], pb[8], va[6], vb[6], val[6], dd[36];
#pragma unroll
    for (int k = 0; k < 8; ++k) { pa[k] = float(c.s.mid[8 * a + k]); pb[k] = float(c.s.mid[8 * b + k]); }
#pragma unroll
    for (int k = 0; k < 6; ++k) { va[k] = float(x[6 * a + k]); vb[k] = float(x[6 * b + k]); }
    joint_jacobian_slice<float>(law, prm, pa, pb, va, vb, c.P.dt, c.P.warp, slice, val, dd);
#pragma unroll
    for (int k = 0; k < 36; ++k) o[k] = dd[k];
  } else {
    double* o = dst ? reinterpret_cast<double*>(dst) : jac_slice<false>(c, q, slice);
    double val[6], dd[36];
    joint_jacobian_slice<double>(law, prm, c.s.mid + 8 * a, c.s.mid + 8 * b, x + 6 * a, x + 6 * b, c.P.dt, c.P.warp,
                                 slice, val, dd);
#pragma unroll
    for (int k = 0; k < 36; ++k) o[k] = dd[k];
    if (write_conn && slice == 0) {
#pragma unroll
      for (int r = 0; r < 6; ++r) c.s.conn[6 * q + r] = val[r];
    }
  }
}

// Joint q at (mid, x): Jacobian slice `slice` with, on slice 0, the joint's value (jac), or the
// value alone (slice 0 only).
template <bool MIXED>
__device__ inline void op_joint(const Ctx& c, const double* x, int q, int slice, bool jac) {
  if (!jac) {
    op_joint_value(c, x, q);
    return;
  }
  op_joint_slice<MIXED>(c, x, q, slice, true);
  if (MIXED && slice == 0) op_joint_value(c, x, q);
}

// Gather + POST (functions::gather_term, body_post) of dynamic node i: mass block, residual and
// its scales; returns the node's worst relative residual^2 (newton.rs:139-151).
__device__ inline double op_post(const Ctx& c, const double* x, double half, int i) {
  double worst = 0.0;
  int q = c.A.dn_body[c.d.dyn_off + i];
  int g = c.gbody(q);
  double tot[6];
  ld_n<6>(c.s.ext + 6 * (size_t)q, tot);
  int p0 = c.A.ib_inc_ptr[c.d.inc_off + q], p1 = c.A.ib_inc_ptr[c.d.inc_off + q + 1];
  for (int t = p0; t < p1; ++t) {
    int ref = c.A.ib_inc_ref[t];
    int jq = ref >> 1;
    double w[6];
    ld_n<6>(c.s.conn + 6 * (size_t)jq, w);
    if (ref & 1) {
#pragma unroll
      for (int k = 0; k < 6; ++k) tot[k] = tot[k] - w[k];
    } else {
#pragma unroll
      for (int k = 0; k < 6; ++k) tot[k] = tot[k] + w[k];
    }
  }
  double I9[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) I9[k] = c.W.inertia[(size_t)k * c.W.n + g];
  const bool diag = c.W.diagonal[g] != 0;
  const double mass = c.W.mass[g];
  double mid[8], inv[8];
  ld_n<8>(c.s.mid + 8 * (size_t)q, mid);
  motor_reverse(mid, inv);
  double blk[36];
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
  st_n<36>(c.s.mass + 36 * (size_t)i, blk);
  double vv[6], p[6], nn[6], hh[6], res[6];
  ld_n<6>(x + 6 * (size_t)q, vv);
  ld_n<6>(c.s.snap + 6 * (size_t)q, nn);
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) acc += blk[r * 6 + k] * vv[k];
    p[r] = acc;
    hh[r] = tot[r] * half;
  }
#pragma unroll
  for (int r = 0; r < 6; ++r) res[r] = -(p[r] - nn[r] - hh[r]);
  st_n<6>(c.s.rhs + 6 * (size_t)i, res);
  auto sq3 = [](const double* v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; };
  double lin = fmax(fmax(fmax(sq3(p), sq3(nn)), sq3(hh)), kFloor2);
  double ang = fmax(fmax(fmax(sq3(p + 3), sq3(nn + 3)), sq3(hh + 3)), kFloor2);
  reinterpret_cast<double2*>(c.s.scale)[i] = make_double2(lin, ang);
  worst = nan_max(worst, sq3(res) / lin);
  worst = nan_max(worst, sq3(res + 3) / ang);
  return worst;
}

// Assembly entry e of cell (node i, kind): kind 0 the diagonal block, 1 (node row, parent col),
// 2 (parent row, node col) (rows/assemble.rs, functions::assemble_term): the mass block (diagonal
// only) then every contributing joint end in joint order with the mid-point factors pf on pose
// columns and vf on velocity columns: pf = -half^2 (times the pose factor scale), vf = -half.
// Writes the entry; *counts says whether it enters ||A||_F.
template <bool MIXED>
__device__ inline double op_assemble(const Ctx& c, double pf, double vf, int cell, int e, bool* counts) {
  int i = cell / 3, kind = cell % 3;
  int r = e / 6, col = e % 6;
  double acc = (kind == 0) ? c.s.mass0[36 * (size_t)i + e] : 0.0;
  int p0 = c.A.cell_ptr[c.d.cell_off + cell], p1 = c.A.cell_ptr[c.d.cell_off + cell + 1];
  for (int k = p0; k < p1; ++k) {
    int term = c.A.cell_terms[k] & ~kTermTorsional;
    int q = term >> 2, re = (term >> 1) & 1, ce = term & 1;
    const auto* jp = jac_slice<MIXED>(c, q, ce);
    const auto* jv = jac_slice<MIXED>(c, q, 2 + ce);
    double pv = double(jp[r * 6 + col]), vv = double(jv[r * 6 + col]);
    if (re) { pv = -pv; vv = -vv; }
    acc = acc + pf * pv + vf * vv;
  }
  double* dst = kind == 0 ? c.s.D : (kind == 1 ? c.s.Acp : c.s.Apc);
  dst[36 * (size_t)i + e] = acc;
  *counts = kind == 0 || c.A.dn_parent[c.d.dyn_off + i] >= 0;
  return acc;
}

// Block t of a block-LU island: the diagonal block of node t (t < m), else an off-diagonal block
// of a slot (Up of slot s at m + 2s, Lo at m + 2s + 1).
__device__ __forceinline__ double* lu_block(const Ctx& c, int t) {
  return t < c.d.m ? c.s.D + 36 * (size_t)t : c.s.G + 36 * (size_t)(t - c.d.m);
}

// Assembly entry e of cell t of a block-LU island: the mass block (diagonal cells) then every
// contributing joint end in cell order, with the factors of op_assemble. Writes the block's entry
// and returns it (every block of such an island enters ||A||_F).
template <bool MIXED>
__device__ inline double op_assemble_lu(const Ctx& c, double pf, double vf, int t, int e) {
  const int r = e / 6, col = e % 6;
  double acc = (t < c.d.m) ? c.s.mass0[36 * (size_t)t + e] : 0.0;
  const int p0 = c.A.cell_ptr[c.d.cell_off + t], p1 = c.A.cell_ptr[c.d.cell_off + t + 1];
  for (int k = p0; k < p1; ++k) {
    int term = c.A.cell_terms[k] & ~kTermTorsional;
    int q = term >> 2, re = (term >> 1) & 1, ce = term & 1;
    const auto* jp = jac_slice<MIXED>(c, q, ce);
    const auto* jv = jac_slice<MIXED>(c, q, 2 + ce);
    double pv = double(jp[r * 6 + col]), vv = double(jv[r * 6 + col]);
    if (re) { pv = -pv; vv = -vv; }
    acc = acc + pf * pv + vf * vv;
  }
  lu_block(c, t)[e] = acc;
  return acc;
}

// trial entry t (body t/6, component t%6) = base + alpha dv on dynamic bodies; kinematic bodies
// keep their prescribed twist.
__device__ inline void op_trial(const Ctx& c, double alpha, int t) {
  int q = t / 6, k = t % 6;
  int i = c.A.ib_order[c.d.body_off + q];
  c.s.trial[t] = (i >= 0) ? c.s.base[t] + c.s.dv[6 * i + k] * alpha : c.s.base[t];
}

// World twist (vm) and world momentum (snap) of island body q at the current state.
__device__ inline void op_load_world_state(const Ctx& c, int q) {
  int g = c.gbody(q);
  double pose[8], mom[6], I9[9];
  local_pose(c, g, pose);
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
  st_n<6>(c.s.vm + 6 * (size_t)q, wv);
  st_n<6>(c.s.snap + 6 * (size_t)q, p6);
}

// External wrench of island body q: gravity (F, p x F) and the uniform field, frozen over the whole
// step.
__device__ inline void op_load_external(const Ctx& c, int q) {
  double e[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int g = c.gbody(q);
  double4 pm = reinterpret_cast<const double4*>(c.W.pos_mass)[g];
  pm.x = pm.x - c.frame[0];  // the moment arm from the island's anchor
  pm.y = pm.y - c.frame[1];
  pm.z = pm.z - c.frame[2];
  if (c.P.splits > 0) {
    int il = g - c.P.wbody_off;
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
  add_uniform_field(c.W.wparams[c.d.world].field_accel, pm, e);
  st_n<6>(c.s.ext + 6 * (size_t)q, e);
}

// commit_span (newton.rs:708-753) for dynamic node i: M = M0 * exp(span v), P = 2 P_mid - P_n
// (P_mid itself when the span did not converge).
__device__ inline void op_commit(const Ctx& c, double span, double half, bool converged, int i) {
  int q = c.A.dn_body[c.d.dyn_off + i];
  int g = c.gbody(q);
  double m0[8], vb[6], e[8], pm[8], inv[8], vbody[6], v6[6], I9[9];
  local_pose(c, g, m0);
#pragma unroll
  for (int k = 0; k < 9; ++k) I9[k] = c.W.inertia[(size_t)k * c.W.n + g];
  double vq[6], snap[6];
  ld_n<6>(c.s.vm + 6 * (size_t)q, vq);
  ld_n<6>(c.s.snap + 6 * (size_t)q, snap);
  screw_from6(vq, vb);
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
  for (int k = 0; k < 6; ++k) pnew[k] = converged ? psm[k] * 2.0 - snap[k] : psm[k];
  double en[8], mnew[8], minv[8], pnb[6], pbody[6], out6[6];
  twist_exp(vb, span, en);
  motor_compose(m0, en, mnew);
  motor_reverse(mnew, minv);
  screw_from6(pnew, pnb);
  wrench_transport(pnb, minv, pbody);
  screw_to6(pbody, out6);
  double mw[8];
  motor_compose(mnew, c.frame + 12, mw);  // back to world coordinates
#pragma unroll
  for (int k = 0; k < 8; ++k) c.W.pose[(size_t)k * c.W.n + g] = mw[k];
#pragma unroll
  for (int k = 0; k < 6; ++k) c.W.mom[(size_t)k * c.W.n + g] = out6[k];
}

// ── warp-cooperative 6x6 block operations of the tree solve ─────────────────
// Inverse by Gauss-Jordan with partial pivoting: lane c < 12 holds column c of [A | I]. Returns
// false (to every lane) if a pivot is zero or not finite.
__device__ inline bool warp_inverse6(const double* a, double* out) {
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
__device__ inline void warp_mm6(const double* A, const double* B, double* C) {
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
__device__ inline void warp_mv6_sub(const double* A, const double* x, double* y) {
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
__device__ inline void warp_mv6(const double* A, const double* x, double* y) {
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

// ── the same block operations for one thread ────────────────────────────────
// Each does per entry exactly the arithmetic of its warp-cooperative counterpart above (same
// operand order, same sums in the same order), so a node solved by one thread matches a node
// solved by one warp bit for bit; a thread holds the whole block in registers, so no shuffles.

// Gauss-Jordan inverse of a (row-major 6x6) with partial pivoting into out. Returns false if a
// pivot is zero or not finite. Only the right half of [A | I] is kept past the column being
// eliminated: the left half's columns to the left of it are never read again.
// STRIDE places entry e of a and of out at [e * STRIDE] (1: plain row-major arrays).
template <int STRIDE = 1>
__device__ __forceinline__ bool thread_inverse6(const double* a, double* out) {
  double M[6][12];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
#pragma unroll
    for (int c = 0; c < 6; ++c) M[r][c] = a[(r * 6 + c) * STRIDE];
#pragma unroll
    for (int c = 0; c < 6; ++c) M[r][6 + c] = (r == c) ? 1.0 : 0.0;
  }
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    int piv = k;
    double best = fabs(M[k][k]);
#pragma unroll
    for (int r = k + 1; r < 6; ++r) {
      double x = fabs(M[r][k]);
      if (x > best) { best = x; piv = r; }
    }
#pragma unroll
    for (int c = k; c < 12; ++c) {  // swap rows k and piv by selects (registers stay registers)
      const double mk = M[k][c];
      double mp = mk;
#pragma unroll
      for (int r = k + 1; r < 6; ++r) mp = (r == piv) ? M[r][c] : mp;
#pragma unroll
      for (int r = k + 1; r < 6; ++r) M[r][c] = (r == piv) ? mk : M[r][c];
      M[k][c] = mp;
    }
    const double pv = M[k][k];
    if (!(fabs(pv) > 0.0) || !isfinite(pv)) ok = false;
    const double ip = 1.0 / pv;
#pragma unroll
    for (int c = k; c < 12; ++c) M[k][c] = M[k][c] * ip;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (r == k) continue;
      const double f = M[r][k];
#pragma unroll
      for (int c = k; c < 12; ++c) M[r][c] = M[r][c] - f * M[k][c];
    }
  }
#pragma unroll
  for (int r = 0; r < 6; ++r)
#pragma unroll
    for (int c = 0; c < 6; ++c) out[(r * 6 + c) * STRIDE] = M[r][6 + c];
  return ok;
}

// ── the mixed path's pivot inverse: Newton-Schulz, FP32 steps and an FP64 correction ──
// With EXG_NEWTON_NS_PIVOT set on a mixed-precision world, each 6x6 pivot block D of the
// elimination is inverted by Newton-Schulz (the reference's iteration, newton.rs:209-327, at block
// size), warm-started like the reference's warm path from the same node's inverse of the
// previous solve in this step, when there is one:
//  1. warm: R = I - D X_prev in FP64; where max|R| <= kNsWarmTol, one FP64 Newton-Schulz
//     correction D^-1 = X_prev + X_prev R (the residual squares) and nothing else;
//  2. otherwise FP32 Newton-Schulz steps held in registers on the symmetrically scaled block
//     B = S D S (s_r = 1/sqrt|d_rr|, 1 where d_rr is zero or not finite, B rounded to FP32):
//     R = I - B X, X <- X + X R, until max|R| <= kNsTol, or until the residual, once below
//     kNsFloor, stops halving (the FP32 floor of a less well conditioned block), at most
//     kNsMaxIter steps; seeded with the scaled previous inverse S^-1 X_prev S^-1 where its FP64
//     residual is below 1/2, else with I where ||I - B||_inf < 1/2, else with the transposed
//     seed B^T / (||B||_1 ||B||_inf), which converges for every non-singular B (the reference's
//     seed_transpose, newton.rs:209-241);
//  3. one FP64 Newton-Schulz correction of X64 = S X S against D: R = I - D X64,
//     D^-1 = X64 + X64 R.
// A block whose FP32 residual ends above kNsAccept (singular, not finite, or too ill-conditioned
// for FP32) takes the FP64 Gauss-Jordan inverse instead. The thread form (a wide elimination
// level) and the warp form (a narrow level, the island kernel) do per entry the same operations
// in the same order with explicitly rounded FMAs, so they give the same bits.
constexpr int kNsMaxIter = 40;
constexpr float kNsTol = 1e-6f;
constexpr float kNsFloor = 1.0f / 64.0f;
constexpr float kNsAccept = 1e-3f;
constexpr float kNsIdentitySeed = 0.5f;
constexpr double kNsWarmTol = 1e-4;
constexpr double kNsWarmSeed = 0.5;

__device__ __forceinline__ double ns_scale(double d) {
  const double a = fabs(d);
  return (a > 0.0 && a < INFINITY) ? 1.0 / sqrt(a) : 1.0;
}
// 0: take another step, 1: stop (converged or at the FP32 floor), -1: failed
__device__ __forceinline__ int ns_verdict(float rmax, bool nan, float prev) {
  if (nan || !(rmax < 1e30f)) return -1;
  if (rmax <= kNsTol) return 1;
  if (rmax < kNsFloor && !(rmax < 0.5f * prev)) return 1;
  return 0;
}

// One thread: out = the inverse of the block a, both row-major with entry e at [e * STRIDE] (a
// thread's two columns of shared memory; they must not overlap). With warm set, out holds on entry
// an earlier inverse (of this block before a small change). Returns false if the block is
// singular (by the Gauss-Jordan fallback's test). *steps receives the FP32 steps taken (0 where
// the warm correction sufficed), or -1 where the block fell back to Gauss-Jordan. The FP32 block
// waits in out's slots while the iteration runs, so registers hold X and R only.
template <int STRIDE>
__device__ __forceinline__ bool thread_ns_inverse6(const double* a, double* out, bool warm, int* steps = nullptr) {
  // volatile reads: a, out and B are read again where needed instead of being held in registers
  const volatile double* av = a;
  volatile double* ov = out;
  bool warm_seed = false;
  if (warm) {
    double R[36];
    double r = 0.0;
    bool nan = false;
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) t = __fma_rn(av[(k * 6 + j) * STRIDE], ov[(j * 6 + c) * STRIDE], t);
        const double v = (k == c ? 1.0 : 0.0) - t;
        R[k * 6 + c] = v;
        const double x = fabs(v);
        nan = nan || (x != x);
        r = x > r ? x : r;
      }
    if (!nan && r <= kNsWarmTol) {  // X_prev + X_prev R, row by row in place
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        double xr[6], o[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) xr[k] = ov[(i * 6 + k) * STRIDE];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          double t = xr[c];
#pragma unroll
          for (int k = 0; k < 6; ++k) t = __fma_rn(xr[k], R[k * 6 + c], t);
          o[c] = t;
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) ov[(i * 6 + c) * STRIDE] = o[c];
      }
      if (steps) *steps = 0;
      return true;
    }
    warm_seed = !nan && r < kNsWarmSeed;
  }
  float* B = reinterpret_cast<float*>(out);  // entry e at B[2 * e * STRIDE]
  const volatile float* Bv = B;
  double s[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) s[r] = ns_scale(a[(r * 7) * STRIDE]);
  float X[36];
  float one = 0.0f, inf = 0.0f, off = 0.0f;
  {
    float colsum[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) colsum[c] = 0.0f;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      float row = 0.0f, rowoff = 0.0f;
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        const int e = r * 6 + c;
        const float v = (float)((a[e * STRIDE] * s[r]) * s[c]);
        X[e] = warm_seed ? (float)((ov[e * STRIDE] / s[r]) / s[c]) : 0.0f;  // read before B takes the slot
        B[2 * e * STRIDE] = v;
        row += fabsf(v);
        rowoff += fabsf((r == c ? 1.0f : 0.0f) - v);
        colsum[c] += fabsf(v);
      }
      inf = fmaxf(inf, row);
      off = fmaxf(off, rowoff);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) one = fmaxf(one, colsum[c]);
  }
  if (!warm_seed) {
    const float sc = 1.0f / (one * inf);
    const bool eye = off < kNsIdentitySeed;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = 0; c < 6; ++c) X[r * 6 + c] = eye ? (r == c ? 1.0f : 0.0f) : Bv[2 * (c * 6 + r) * STRIDE] * sc;
  }
  float prev = INFINITY, rmax = INFINITY;
  int verdict = 0, it = 0;
#pragma unroll 1
  for (; it < kNsMaxIter; ++it) {
    float R[36];
    bool nan = false;
    rmax = 0.0f;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      float br[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) br[k] = Bv[2 * (r * 6 + k) * STRIDE];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        float t = 0.0f;
#pragma unroll
        for (int k = 0; k < 6; ++k) t = __fmaf_rn(br[k], X[k * 6 + c], t);
        const float v = (r == c ? 1.0f : 0.0f) - t;
        R[r * 6 + c] = v;
        const float x = fabsf(v);
        nan = nan || (x != x);
        rmax = x > rmax ? x : rmax;
      }
    }
    verdict = ns_verdict(rmax, nan, prev);
    if (verdict != 0) break;
    prev = rmax;
    // X <- X + X R, row by row in place: row r of the new X reads only row r of the old one
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      float xr[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        float t = X[r * 6 + c];
#pragma unroll
        for (int k = 0; k < 6; ++k) t = __fmaf_rn(X[r * 6 + k], R[k * 6 + c], t);
        xr[c] = t;
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) X[r * 6 + c] = xr[c];
    }
  }
  if (!(verdict == 1 && rmax <= kNsAccept)) {
    if (steps) *steps = -1;
    return thread_inverse6<STRIDE>(a, out);
  }
  if (steps) *steps = it;
  // the FP64 correction, one column at a time: q = e_c - D x_c, then column c of X64 + X64 q
  double xd[36];
#pragma unroll
  for (int r = 0; r < 6; ++r)
#pragma unroll
    for (int c = 0; c < 6; ++c) xd[r * 6 + c] = ((double)X[r * 6 + c] * s[r]) * s[c];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double q[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) t = __fma_rn(av[(k * 6 + j) * STRIDE], xd[j * 6 + c], t);
      q[k] = (k == c ? 1.0 : 0.0) - t;
    }
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double t = xd[r * 6 + c];
#pragma unroll
      for (int k = 0; k < 6; ++k) t = __fma_rn(xd[r * 6 + k], q[k], t);
      out[(r * 6 + c) * STRIDE] = t;
    }
  }
  return true;
}

// Entry idx of a block held two entries per lane (entry e in lane e, entries 32..35 in the second
// register of lanes 0..3); every lane of the warp calls it.
__device__ __forceinline__ float ns_get(float v0, float v1, int idx) {
  const float x = __shfl_sync(0xffffffffu, v0, idx & 31);
  const float y = __shfl_sync(0xffffffffu, v1, idx & 31);
  return idx < 32 ? x : y;
}
__device__ __forceinline__ double ns_get(double v0, double v1, int idx) {
  const double x = __shfl_sync(0xffffffffu, v0, idx & 31);
  const double y = __shfl_sync(0xffffffffu, v1, idx & 31);
  return idx < 32 ? x : y;
}
__device__ __forceinline__ float ns_warp_max(float m) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  return m;
}
__device__ __forceinline__ double ns_warp_max(double m) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  return m;
}

// One warp: out = the inverse of the row-major block a (both in memory, not overlapping), the
// same bits as thread_ns_inverse6; with warm set, out holds on entry an earlier inverse. Returns
// false (to every lane) if the block is singular.
__device__ inline bool warp_ns_inverse6(const double* a, double* out, bool warm, int* steps = nullptr) {
  const int lane = threadIdx.x & 31;
  const bool has1 = lane < 4;
  const int e0 = lane, e1 = has1 ? lane + 32 : lane;  // lanes 4.. repeat e0 in their second slot
  const int r0 = e0 / 6, c0 = e0 % 6, r1 = e1 / 6, c1 = e1 % 6;
  bool warm_seed = false;
  if (warm) {
    double t0 = 0.0, t1 = 0.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      t0 = __fma_rn(a[r0 * 6 + j], out[j * 6 + c0], t0);
      t1 = __fma_rn(a[r1 * 6 + j], out[j * 6 + c1], t1);
    }
    const double R0 = (r0 == c0 ? 1.0 : 0.0) - t0, R1 = (r1 == c1 ? 1.0 : 0.0) - t1;
    const double x0 = fabs(R0), x1 = has1 ? fabs(R1) : 0.0;
    const bool nan = __any_sync(0xffffffffu, (x0 != x0) || (x1 != x1));
    const double r = ns_warp_max(x1 > x0 ? x1 : x0);
    if (!nan && r <= kNsWarmTol) {  // X_prev + X_prev R
      double o0 = out[e0], o1 = out[e1];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        o0 = __fma_rn(out[r0 * 6 + k], ns_get(R0, R1, k * 6 + c0), o0);
        o1 = __fma_rn(out[r1 * 6 + k], ns_get(R0, R1, k * 6 + c1), o1);
      }
      __syncwarp();
      out[e0] = o0;
      if (has1) out[e1] = o1;
      __syncwarp();
      if (steps && lane == 0) *steps = 0;
      return true;
    }
    warm_seed = !nan && r < kNsWarmSeed;
  }
  const double sr0 = ns_scale(a[r0 * 7]), sc0 = ns_scale(a[c0 * 7]);
  const double sr1 = ns_scale(a[r1 * 7]), sc1 = ns_scale(a[c1 * 7]);
  const float B0 = (float)((a[e0] * sr0) * sc0), B1 = (float)((a[e1] * sr1) * sc1);
  float X0, X1;
  if (warm_seed) {
    X0 = (float)((out[e0] / sr0) / sc0);
    X1 = (float)((out[e1] / sr1) / sc1);
  } else {
    float one = 0.0f, inf = 0.0f, off = 0.0f;
    {
      const int i = lane % 6;
      float row = 0.0f, col = 0.0f, rowoff = 0.0f;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const float v = ns_get(B0, B1, i * 6 + j);
        row += fabsf(v);
        rowoff += fabsf((i == j ? 1.0f : 0.0f) - v);
        col += fabsf(ns_get(B0, B1, j * 6 + i));
      }
      if (lane >= 6) row = col = rowoff = 0.0f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        row = fmaxf(row, __shfl_xor_sync(0xffffffffu, row, o));
        col = fmaxf(col, __shfl_xor_sync(0xffffffffu, col, o));
        rowoff = fmaxf(rowoff, __shfl_xor_sync(0xffffffffu, rowoff, o));
      }
      inf = row;
      one = col;
      off = rowoff;
    }
    const float sc = 1.0f / (one * inf);
    const bool eye = off < kNsIdentitySeed;
    X0 = eye ? (r0 == c0 ? 1.0f : 0.0f) : ns_get(B0, B1, c0 * 6 + r0) * sc;
    X1 = eye ? (r1 == c1 ? 1.0f : 0.0f) : ns_get(B0, B1, c1 * 6 + r1) * sc;
  }
  float prev = INFINITY, rmax = INFINITY;
  int verdict = 0, it = 0;
#pragma unroll 1
  for (; it < kNsMaxIter; ++it) {
    float t0 = 0.0f, t1 = 0.0f;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float b0 = ns_get(B0, B1, r0 * 6 + k), x0 = ns_get(X0, X1, k * 6 + c0);
      const float b1 = ns_get(B0, B1, r1 * 6 + k), x1 = ns_get(X0, X1, k * 6 + c1);
      t0 = __fmaf_rn(b0, x0, t0);
      t1 = __fmaf_rn(b1, x1, t1);
    }
    const float R0 = (r0 == c0 ? 1.0f : 0.0f) - t0, R1 = (r1 == c1 ? 1.0f : 0.0f) - t1;
    const float a0 = fabsf(R0), a1 = has1 ? fabsf(R1) : 0.0f;
    const bool nan = __any_sync(0xffffffffu, (a0 != a0) || (a1 != a1));
    rmax = ns_warp_max(a1 > a0 ? a1 : a0);
    verdict = ns_verdict(rmax, nan, prev);
    if (verdict != 0) break;
    prev = rmax;
    float n0 = X0, n1 = X1;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      n0 = __fmaf_rn(ns_get(X0, X1, r0 * 6 + k), ns_get(R0, R1, k * 6 + c0), n0);
      n1 = __fmaf_rn(ns_get(X0, X1, r1 * 6 + k), ns_get(R0, R1, k * 6 + c1), n1);
    }
    X0 = n0;
    X1 = n1;
  }
  if (!(verdict == 1 && rmax <= kNsAccept)) {
    if (steps && lane == 0) *steps = -1;
    __syncwarp();
    return warp_inverse6(a, out);
  }
  if (steps && lane == 0) *steps = it;
  const double xd0 = ((double)X0 * sr0) * sc0, xd1 = ((double)X1 * sr1) * sc1;
  double q0 = 0.0, q1 = 0.0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const double g0 = ns_get(xd0, xd1, j * 6 + c0), g1 = ns_get(xd0, xd1, j * 6 + c1);
    q0 = __fma_rn(a[r0 * 6 + j], g0, q0);
    q1 = __fma_rn(a[r1 * 6 + j], g1, q1);
  }
  const double Q0 = (r0 == c0 ? 1.0 : 0.0) - q0, Q1 = (r1 == c1 ? 1.0 : 0.0) - q1;
  double o0 = xd0, o1 = xd1;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    o0 = __fma_rn(ns_get(xd0, xd1, r0 * 6 + k), ns_get(Q0, Q1, k * 6 + c0), o0);
    o1 = __fma_rn(ns_get(xd0, xd1, r1 * 6 + k), ns_get(Q0, Q1, k * 6 + c1), o1);
  }
  __syncwarp();
  out[e0] = o0;
  if (has1) out[e1] = o1;
  __syncwarp();
  return true;
}

// The pivot inverse of the elimination: on the mixed path with Newton-Schulz pivots selected (ns),
// warp_ns_inverse6 (warm: out holds the node's inverse from the previous solve of this step);
// otherwise FP64 Gauss-Jordan.
template <bool MIXED>
__device__ __forceinline__ bool warp_pivot_inverse6(const double* a, double* out, bool ns, bool warm) {
  if (MIXED && ns) return warp_ns_inverse6(a, out, warm);
  return warp_inverse6(a, out);
}

// ── scalar helpers of the span budget ───────────────────────────────────────
__device__ inline bool log2_floor(double v, int* e) {
  if (!(v > 0.0)) return false;
  double x = v;
  int k = 0;
  while (x >= 2.0) { x /= 2.0; ++k; if (k > 250) return false; }
  while (x < 1.0 && k > -250) { x *= 2.0; --k; }
  *e = k;
  return true;
}
__device__ inline int div_euclid(int a, int b) { int q = a / b; if (a % b < 0) q -= 1; return q; }

// signal_log2 (newton.rs:812-861) from ||A||_F^2 and the mass blocks' ||M||_F^2.
__device__ inline bool signal_from_norms(bool assembled, double a_norm2, double massn, int* r) {
  if (!assembled) return false;
  double stiff = ScalarTraits<double>::eff_zero(massn) ? 0.0 : a_norm2 / massn;
  return log2_floor(stiff, r);
}

}  // namespace exg_newton
