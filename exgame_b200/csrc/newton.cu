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
#include <set>
#include "body.cuh"
#include "newton_ops.cuh"

namespace {

using namespace exg_newton;

#ifndef EXG_NEWTON_MIN_BLOCKS
#define EXG_NEWTON_MIN_BLOCKS 1  // CTAs per SM the register budget is sized for
#endif
#ifndef EXG_NEWTON_THREADS
#define EXG_NEWTON_THREADS 256
#endif
constexpr int kThreads = EXG_NEWTON_THREADS;
constexpr int kMinBlocks = EXG_NEWTON_MIN_BLOCKS;
constexpr int kWarps = kThreads / 32;

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

// ── phases: the island's items spread over the CTA ──────────────────────────
__device__ void phase_pre(const Ctx& c, const double* v, double half) {
  for (int q = threadIdx.x; q < c.d.nb; q += blockDim.x) op_pre(c, v, half, q);
}

template <bool MIXED>
__device__ void phase_joints(const Ctx& c, const double* v, bool jac) {
  if (jac) {
    // a warp takes 16 joints and one kind of slice (pose 0, 1 or twist 2, 3), so it follows one path
    const int total = 64 * ((c.d.nj + 15) / 16);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int w = t >> 5, l = t & 31, q = (w >> 1) * 16 + (l >> 1);
      if (q < c.d.nj) op_joint<MIXED>(c, v, q, 2 * (w & 1) + (l & 1), true);
    }
  } else {
    for (int q = threadIdx.x; q < c.d.nj; q += blockDim.x) op_joint<MIXED>(c, v, q, 0, false);
  }
}

__device__ double phase_post(const Ctx& c, const double* v, double half, double* red) {
  double worst = 0.0;
  for (int i = threadIdx.x; i < c.d.m; i += blockDim.x) worst = nan_max(worst, op_post(c, v, half, i));
  return block_max(worst, red);
}

__device__ void copy_mass0(const Ctx& c) {
  for (int t = threadIdx.x; t < 36 * c.d.m; t += blockDim.x) c.s.mass0[t] = c.s.mass[t];
}

// Returns ||A||_F^2.
template <bool MIXED>
__device__ double phase_assemble(const Ctx& c, double half, double* red) {
  double sumsq = 0.0;
  const double pf = -(half * half) * c.P.pose_factor_scale, vf = -half;
  if (c.d.solver == 1) {
    const int cells = c.d.m + 2 * c.d.n_slots;
    for (int t = threadIdx.x; t < cells * 36; t += blockDim.x) {
      const double acc = op_assemble_lu<MIXED>(c, pf, vf, t / 36, t % 36);
      sumsq += acc * acc;
    }
    return block_sum(sumsq, red);
  }
  const int cells = 3 * c.d.m;
  for (int t = threadIdx.x; t < cells * 36; t += blockDim.x) {
    bool counts;
    double acc = op_assemble<MIXED>(c, pf, vf, t / 36, t % 36, &counts);
    if (counts) sumsq += acc * acc;
  }
  return block_sum(sumsq, red);
}

// Exact solve of A dv = rhs by block LU on the island's elimination order (solver 1: dynamic
// cycles). Level by level from the first eliminated nodes (left-looking: a node's row, column and
// diagonal blocks receive every product of the lower levels in a fixed order, one warp per target
// block), then per node the pivot inverse D^-1 and the scaled column S = A(j, k) D_k^-1 in place;
// the right-hand side follows the same updates (b_k -= S_kp y_p). Back substitution from the last
// level: x_k = D_k^-1 (y_k - sum_j A(k, j) x_j). Returns false if a pivot block is singular (dv is
// then NaN, which the line search rejects).
template <bool MIXED, bool NS>
__device__ bool phase_solve_lu(const Ctx& c, int* flag, bool warm) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m = c.d.m;
  const int* lv = c.A.lv_ptr + c.d.lv_off;
  const int* nodes = c.A.lv_nodes + c.d.dyn_off;
  const int* lg = c.A.gn_lgrp + c.d.gen_lv_off;
  const int* rp = c.A.gn_rop_ptr + c.d.gen_off;
  const int* sp = c.A.gn_slot_ptr + c.d.gen_off;
  const int* scol = c.A.gn_slot_col + c.d.gen_slot_off;
  if (threadIdx.x == 0) *flag = 1;
  for (int t = threadIdx.x; t < 6 * m; t += blockDim.x) c.s.bvec[t] = c.s.rhs[t];
  __syncthreads();
  for (int L = 0; L < c.d.n_levels; ++L) {
    for (int g = lg[L] + warp; g < lg[L + 1]; g += kWarps) {
      const int4 G = c.A.gn_grp[g];
      double* tgt = lu_block(c, G.x);
      for (int o = G.y; o < G.z; ++o) {
        const int2 op = c.A.gn_ops[o];
        warp_mm6<true>(lu_block(c, op.x), lu_block(c, op.y), tgt);
      }
    }
    for (int u = lv[L] + warp; u < lv[L + 1]; u += kWarps) {
      const int k = nodes[u];
      for (int t = rp[k]; t < rp[k + 1]; ++t) {
        const int2 op = c.A.gn_rops[t];
        warp_mv6_sub(lu_block(c, op.x), c.s.bvec + 6 * (size_t)op.y, c.s.bvec + 6 * (size_t)k);
      }
    }
    __syncthreads();
    for (int u = lv[L] + warp; u < lv[L + 1]; u += kWarps) {
      const int k = nodes[u];
      const bool ok = warp_pivot_inverse6<MIXED && NS>(lu_block(c, k), c.s.Dinv + 36 * (size_t)k, c.P.ns_pivot, warm);
      if (!ok && lane == 0) *flag = 0;
      for (int s = sp[k]; s < sp[k + 1]; ++s) {
        double* lo = c.s.G + 72 * (size_t)s + 36;
        warp_mm6<false>(lo, c.s.Dinv + 36 * (size_t)k, lo);
      }
    }
    __syncthreads();
  }
  for (int L = c.d.n_levels - 1; L >= 0; --L) {
    for (int u = lv[L] + warp; u < lv[L + 1]; u += kWarps) {
      const int k = nodes[u];
      for (int s = sp[k]; s < sp[k + 1]; ++s)
        warp_mv6_sub(c.s.G + 72 * (size_t)s, c.s.dv + 6 * (size_t)scol[s], c.s.bvec + 6 * (size_t)k);
      warp_mv6(c.s.Dinv + 36 * (size_t)k, c.s.bvec + 6 * (size_t)k, c.s.dv + 6 * (size_t)k);
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

// Exact solve of A dv = rhs on the island's elimination forest. Returns false if a pivot
// block is singular (dv is then NaN, which the line search rejects).
// warm: every node's Dinv slot holds its inverse from an earlier solve of this step (the mixed
// path's Newton-Schulz pivots start from it).
template <bool MIXED, bool NS>
__device__ bool phase_solve(const Ctx& c, int* flag, bool warm) {
  if (c.d.solver == 1) return phase_solve_lu<MIXED, NS>(c, flag, warm);
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
      bool ok = warp_pivot_inverse6<MIXED && NS>(c.s.D + 36 * (size_t)i, c.s.Dinv + 36 * (size_t)i, c.P.ns_pivot, warm);
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
    bool ok = warp_pivot_inverse6<MIXED && NS>(c.s.D + 36 * (size_t)i, c.s.Dinv + 36 * (size_t)i, c.P.ns_pivot, warm);
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

__device__ void make_trial(const Ctx& c, double alpha) {
  for (int t = threadIdx.x; t < 6 * c.d.nb; t += blockDim.x) op_trial(c, alpha, t);
}

__device__ void load_world_state(const Ctx& c) {
  for (int q = threadIdx.x; q < c.d.nb; q += blockDim.x) op_load_world_state(c, q);
}

__device__ void load_external(const Ctx& c) {
  for (int q = threadIdx.x; q < c.d.nb; q += blockDim.x) op_load_external(c, q);
}

struct SolveOut { bool converged; double best; bool assembled; double a_norm2; };

template <bool MIXED, bool NS>
__device__ SolveOut newton_solve(const Ctx& c, double half, double* red, int* flag, int* iters, PhaseTimer& tm,
                                bool* warm) {
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
    o.a_norm2 = phase_assemble<MIXED>(c, half, red);
    o.assembled = true;
    tm.lap(PH_ASSEMBLE);
    phase_solve<MIXED, NS>(c, flag, *warm);
    *warm = true;
    tm.lap(PH_SOLVE);
    // no correction at all -> hand over to sub-division (newton.rs:449-456)
    int nz = 0;
    for (int t = threadIdx.x; t < 6 * c.d.m; t += blockDim.x) nz |= (c.s.dv[t] != 0.0);
    if (!__syncthreads_or(nz)) break;
    copy_bodies6(c, c.s.vm, c.s.base);
    __syncthreads();
    int accepted = -1;
    double alpha = 1.0;
    for (int lane = 0; lane < kLineSearchLanes; ++lane) {
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

__device__ bool signal_log2(const Ctx& c, const SolveOut& o, double* red, int* r) {
  if (!o.assembled) return false;
  double s = 0.0;
  for (int t = threadIdx.x; t < 36 * c.d.m; t += blockDim.x) s += c.s.mass0[t] * c.s.mass0[t];
  double massn = block_sum(s, red);
  return signal_from_norms(o.assembled, o.a_norm2, massn, r);
}

__device__ void commit_span(const Ctx& c, double span, double half, bool converged) {
  for (int i = threadIdx.x; i < c.d.m; i += blockDim.x) op_commit(c, span, half, converged, i);
}

template <bool MIXED, bool NS>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_newton_step(NewtonDeviceArrays A, WorldRef W, const int* __restrict__ queue,
                                                         int n_islands, int* __restrict__ head) {
  __shared__ double red[kWarps];
  __shared__ double frame[kFrameDoubles];
  __shared__ double frame_sh[4 * kFrameThreads];
  static_assert(kThreads == kFrameThreads, "the island frame sums over a CTA of kFrameThreads threads");
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
    const int island = queue[k];
    if (!W.w_active[A.desc[island].world]) continue;  // the world holds this step
    Ctx c = make_ctx(A, W, island);
    island_frame(A, W, c.d, frame_sh, frame);  // the step's frame: the island's centre of mass
    c.frame = frame;
    load_external(c);
    __syncthreads();
    unsigned long long remaining = 1ull << kMaxDepth;
    int depth = 0, spans = 0, iters = 0, maxdepth = 0;
    double last_best = 0.0;
    bool warm = false;  // no solve of this step has filled the Dinv slots yet
    while (remaining > 0) {
      unsigned long long units = 1ull << (kMaxDepth - depth);
      while (units > remaining) { ++depth; units >>= 1; }
      double span = c.P.dt;
      for (int t = 0; t < depth; ++t) span = span / 2.0;
      double half = span / 2.0;
      ++spans;
      maxdepth = max(maxdepth, depth);
      SolveOut o = newton_solve<MIXED, NS>(c, half, red, &flag, &iters, tm, &warm);
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
namespace {
// Block LU plan of an island whose dynamic bodies form cycles. The elimination order is minimum
// degree on the dynamic adjacency (ties to the lowest node), eliminating a node joining its
// remaining neighbours into a clique (the fill). later[k] are k's neighbours eliminated after it
// in the filled graph (by position); the elimination tree's parent is the first of them, and a
// node's level is its height in that tree, so every node a node depends on sits on a lower level.
struct BlockLuPlan {
  std::vector<int> pos, parent, level, slot_first;
  std::vector<std::vector<int>> later, contrib;  // contrib[k]: the p with k in later[p], by position
  int n_levels = 0, n_slots = 0;
  int slot(int k, int j) const {  // the slot of the pair (k, j), j in later[k]
    const std::vector<int>& L = later[k];
    int lo = 0, hi = (int)L.size();
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      if (pos[L[mid]] < pos[j]) lo = mid + 1; else hi = mid;
    }
    return slot_first[k] + lo;
  }
  bool has(int k, int j) const {
    int s = slot(k, j) - slot_first[k];
    return s < (int)later[k].size() && later[k][s] == j;
  }
};

void plan_block_lu(int m, const std::vector<std::vector<int>>& adj, BlockLuPlan& P) {
  std::vector<std::set<int>> nb(m);
  for (int i = 0; i < m; ++i) nb[i].insert(adj[i].begin(), adj[i].end());
  std::set<std::pair<int, int>> queue;  // (current degree, node)
  for (int i = 0; i < m; ++i) queue.insert({(int)nb[i].size(), i});
  P.pos.assign(m, -1);
  P.later.assign(m, {});
  std::vector<int> order;
  order.reserve(m);
  for (int step = 0; step < m; ++step) {
    const int v = queue.begin()->second;
    queue.erase(queue.begin());
    P.pos[v] = step;
    order.push_back(v);
    std::vector<int> ns(nb[v].begin(), nb[v].end());
    P.later[v] = ns;
    for (int u : ns) {
      queue.erase({(int)nb[u].size(), u});
      nb[u].erase(v);
    }
    for (size_t a = 0; a < ns.size(); ++a)
      for (size_t b = a + 1; b < ns.size(); ++b) {
        nb[ns[a]].insert(ns[b]);
        nb[ns[b]].insert(ns[a]);
      }
    for (int u : ns) queue.insert({(int)nb[u].size(), u});
    nb[v].clear();
  }
  for (int k = 0; k < m; ++k)
    std::sort(P.later[k].begin(), P.later[k].end(), [&](int a, int b) { return P.pos[a] < P.pos[b]; });
  P.parent.assign(m, -1);
  P.level.assign(m, 0);
  P.n_levels = m > 0 ? 1 : 0;
  for (int v : order) {
    if (P.later[v].empty()) continue;
    const int p = P.later[v][0];
    P.parent[v] = p;
    P.level[p] = std::max(P.level[p], P.level[v] + 1);
    P.n_levels = std::max(P.n_levels, P.level[p] + 1);
  }
  P.slot_first.assign(m + 1, 0);
  for (int k = 0; k < m; ++k) P.slot_first[k + 1] = P.slot_first[k] + (int)P.later[k].size();
  P.n_slots = P.slot_first[m];
  P.contrib.assign(m, {});
  for (int v : order)
    for (int j : P.later[v]) P.contrib[j].push_back(v);
}
}  // namespace

long long newton_footprint_bytes(int nb, int nj) {
  // scratch, then the structure: 13 ints per body (body list, order, incidence pointers,
  // dynamic list, parents, levels, children, 3 assembly cells), 9 per joint plus its 10 params
  return ((scratch_doubles(nb, nj, nb) + 31) & ~31LL) * 8 + (long long)nb * 13 * 4 + (long long)nj * (9 * 4 + 80) +
         (long long)sizeof(IslandDesc) + 64;
}

NewtonWorld::~NewtonWorld() {
  if (wave_graph_) cudaGraphExecDestroy(wave_graph_);
  if (fork_) cudaEventDestroy(fork_);
  if (join_) cudaEventDestroy(join_);
  if (side_) cudaStreamDestroy(side_);
  for (DevArr<int>* a : {&dw_isl_, &dw_dyn_first_, &dw_live_, &dw_seg_, &dw_act_, &dw_pre_}) a->release();
  for (DevArr<int2>* a : {&dw_body_, &dw_dyn_, &dw_joint_, &dw_cell_, &dw_level_, &dw_cell_terms_}) a->release();
  dw_ctl_.release();
  dw_nodesq_.release();
  dw_desc_.release();
  d_desc.release();
  for (DevArr<int>* a : {&d_isl_body, &d_jl_law, &d_jl_a, &d_jl_b, &d_ib_order, &d_ib_inc_ptr, &d_ib_inc_ref, &d_dn_body,
                         &d_dn_parent, &d_lv_ptr, &d_lv_nodes, &d_ch_ptr, &d_ch_idx, &d_cell_ptr, &d_cell_terms, &d_stats,
                         &d_queue})
    a->release();
  d_jl_params.release();
  for (DevArr<int>* a : {&d_gn_lgrp, &d_gn_rop_ptr, &d_gn_slot_ptr, &d_gn_slot_col}) a->release();
  d_gn_grp.release();
  d_gn_ops.release();
  d_gn_rops.release();
  d_scratch.release();
  d_residual.release();
  d_phase.release();
}

namespace {
// Stage kernels of exg_pivot_inverse: the elimination's pivot inverse on caller-given blocks,
// one thread per block (a wide level's form: the block staged in the thread's column of shared
// memory, as k_w_solve_down does) or one warp per block (a narrow level's and the island kernel's).
constexpr int kPivotThreads = 64;
template <bool MIXED>
__global__ void __launch_bounds__(kPivotThreads) k_pivot_thread(const double* blocks, int n, double* out, int* steps,
                                                                int* singular, bool warm) {
  extern __shared__ double col_base[];
  double* col = col_base + threadIdx.x;
  for (long long b = blockIdx.x * (long long)kPivotThreads + threadIdx.x; b < n;
       b += (long long)gridDim.x * kPivotThreads) {
    const double* a = blocks + 36 * b;
    bool ok;
    int st = 0;
    if (MIXED) {
      for (int e = 0; e < 36; ++e) col[e * kPivotThreads] = a[e];
      if (warm)
        for (int e = 0; e < 36; ++e) col[(36 + e) * kPivotThreads] = out[36 * b + e];
      ok = thread_ns_inverse6<kPivotThreads>(col, col + 36 * kPivotThreads, warm, &st);
      for (int e = 0; e < 36; ++e) out[36 * b + e] = col[(36 + e) * kPivotThreads];
    } else {
      double m[36], inv[36];
      for (int e = 0; e < 36; ++e) m[e] = a[e];
      ok = thread_inverse6(m, inv);
      for (int e = 0; e < 36; ++e) out[36 * b + e] = inv[e];
    }
    if (steps) steps[b] = st;
    if (!ok) atomicOr(singular, 1);
  }
}
template <bool MIXED>
__global__ void __launch_bounds__(kPivotThreads) k_pivot_warp(const double* blocks, int n, double* out, int* steps,
                                                              int* singular, bool warm) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (kPivotThreads / 32);
  for (long long b = (blockIdx.x * (long long)kPivotThreads + threadIdx.x) >> 5; b < n; b += warps) {
    int st = 0;
    const bool ok = MIXED ? warp_ns_inverse6(blocks + 36 * b, out + 36 * b, warm, &st)
                          : warp_inverse6(blocks + 36 * b, out + 36 * b);
    if (steps && lane == 0) steps[b] = st;
    if (!ok && lane == 0) atomicOr(singular, 1);
  }
}
}  // namespace

int launch_pivot_inverse(exg_device_s* dev, const double* blocks, int n, int mixed, int form, int warm, double* out,
                         int* steps, int* singular, cudaStream_t s) {
  const int max_grid = std::max(1, dev->sm_count) * 8;
  if (form == 0) {
    const int grid = (int)std::min<long long>(max_grid, (n + kPivotThreads - 1) / kPivotThreads);
    if (mixed) k_pivot_thread<true><<<grid, kPivotThreads, 72 * kPivotThreads * sizeof(double), s>>>(blocks, n, out,
                                                                                                   steps, singular, warm != 0);
    else k_pivot_thread<false><<<grid, kPivotThreads, 0, s>>>(blocks, n, out, steps, singular, false);
  } else {
    const int grid = (int)std::min<long long>(max_grid, (32LL * n + kPivotThreads - 1) / kPivotThreads);
    if (mixed) k_pivot_warp<true><<<grid, kPivotThreads, 0, s>>>(blocks, n, out, steps, singular, warm != 0);
    else k_pivot_warp<false><<<grid, kPivotThreads, 0, s>>>(blocks, n, out, steps, singular, false);
  }
  EXG_CUDA_TRY(cudaGetLastError());
  return EXG_OK;
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
  h_jl_id.clear();
  for (std::vector<int>* v : {&h_gn_lgrp, &h_gn_rop_ptr, &h_gn_slot_ptr, &h_gn_slot_col}) v->clear();
  h_gn_grp.clear();
  h_gn_ops.clear();
  h_gn_rops.clear();
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
  for (DevArr<int>* a : {&d_gn_lgrp, &d_gn_rop_ptr, &d_gn_slot_ptr, &d_gn_slot_col}) a->size = 0;
  d_gn_grp.size = 0;
  d_gn_ops.size = 0;
  d_gn_rops.size = 0;
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
  std::vector<int> s_jl_id, s_gn_lgrp, s_gn_rop_ptr, s_gn_slot_ptr, s_gn_slot_col;
  std::vector<int4> s_gn_grp;
  std::vector<int2> s_gn_ops, s_gn_rops;
  const int base_gn_lgrp = (int)h_gn_lgrp.size(), base_gn_ptr = (int)h_gn_rop_ptr.size(),
            base_gn_slot = (int)h_gn_slot_col.size(), base_gn_grp = (int)h_gn_grp.size(),
            base_gn_ops = (int)h_gn_ops.size(), base_gn_rops = (int)h_gn_rops.size();
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
      s_jl_id.push_back(J[q]);
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
    d.solver = 0;
    d.n_slots = 0;
    d.gen_off = d.gen_lv_off = d.gen_slot_off = 0;
    if (edges != m - comps) {
      // a cycle among the dynamic bodies: block LU on a minimum-degree order with fill
      BlockLuPlan P;
      plan_block_lu(m, adj, P);
      d.solver = 1;
      d.n_slots = P.n_slots;
      d.n_levels = P.n_levels;
      d.lv_off = base_lv + (int)s_lv_ptr.size();
      std::vector<std::vector<int>> by(P.n_levels);
      for (int i = 0; i < m; ++i) by[P.level[i]].push_back(i);
      {
        int acc = 0;
        for (int L = 0; L < P.n_levels; ++L) {
          s_lv_ptr.push_back(acc);
          for (int i : by[L]) s_lv_nodes.push_back(i);
          acc += (int)by[L].size();
        }
        s_lv_ptr.push_back(acc);
      }
      {  // children of the elimination tree (for the structure read-back; the solve reads gn_*)
        std::vector<std::vector<int>> ch(m);
        for (int i = 0; i < m; ++i) if (P.parent[i] >= 0) ch[P.parent[i]].push_back(i);
        for (int i = 0; i < m; ++i) {
          s_ch_ptr.push_back(base_ch_idx + (int)s_ch_idx.size());
          for (int x : ch[i]) s_ch_idx.push_back(x);
        }
        for (int i = 0; i < m; ++i) { s_dn_body.push_back(dyn_body[i]); s_dn_parent.push_back(P.parent[i]); }
      }
      // update groups per level: a group is one target block of a node and the ordered products
      // subtracted from it (left-looking: every contribution comes from a lower level)
      d.gen_lv_off = base_gn_lgrp + (int)s_gn_lgrp.size();
      d.gen_off = base_gn_ptr + (int)s_gn_rop_ptr.size();
      d.gen_slot_off = base_gn_slot + (int)s_gn_slot_col.size();
      auto up_blk = [&](int k, int j) { return m + 2 * P.slot(k, j); };
      auto lo_blk = [&](int k, int j) { return m + 2 * P.slot(k, j) + 1; };
      for (int L = 0; L < P.n_levels; ++L) {
        s_gn_lgrp.push_back(base_gn_grp + (int)s_gn_grp.size());
        for (int k : by[L]) {
          auto group = [&](int target, const std::vector<int2>& ops) {
            if (ops.empty()) return;
            const int first = base_gn_ops + (int)s_gn_ops.size();
            s_gn_ops.insert(s_gn_ops.end(), ops.begin(), ops.end());
            s_gn_grp.push_back(make_int4(target, first, first + (int)ops.size(), k));
          };
          std::vector<int2> ops;
          for (int p : P.contrib[k]) ops.push_back(make_int2(lo_blk(p, k), up_blk(p, k)));  // D_k -= S_kp A_pk
          group(k, ops);
          for (int j : P.later[k]) {
            std::vector<int2> opu, opl;
            for (int p : P.contrib[k]) {
              if (!P.has(p, j)) continue;
              opu.push_back(make_int2(lo_blk(p, k), up_blk(p, j)));  // A_kj -= S_kp A_pj
              opl.push_back(make_int2(lo_blk(p, j), up_blk(p, k)));  // A_jk -= S_jp A_pk
            }
            group(up_blk(k, j), opu);
            group(lo_blk(k, j), opl);
          }
        }
      }
      s_gn_lgrp.push_back(base_gn_grp + (int)s_gn_grp.size());
      for (int k = 0; k < m; ++k) {
        s_gn_rop_ptr.push_back(base_gn_rops + (int)s_gn_rops.size());
        for (int p : P.contrib[k]) s_gn_rops.push_back(make_int2(lo_blk(p, k), p));  // b_k -= S_kp y_p
        s_gn_slot_ptr.push_back(P.slot_first[k]);
        for (int j : P.later[k]) s_gn_slot_col.push_back(j);
      }
      s_gn_rop_ptr.push_back(base_gn_rops + (int)s_gn_rops.size());
      s_gn_slot_ptr.push_back(P.slot_first[m]);
      // assembly cells: the diagonal blocks, then both blocks of every slot (fill slots get none)
      d.cell_off = base_cell_ptr + (int)s_cell_ptr.size();
      {
        const int n_cells = m + 2 * P.n_slots;
        std::vector<std::vector<int>> cells(n_cells);
        for (int q = 0; q < d.nj; ++q) {
          int ends[2] = {order[s_jl_a[jl0 + q]], order[s_jl_b[jl0 + q]]};
          for (int re = 0; re < 2; ++re) {
            if (ends[re] < 0) continue;
            for (int ce = 0; ce < 2; ++ce) {
              if (ends[ce] < 0) continue;
              const int row = ends[re], col = ends[ce];
              int target;
              if (row == col) target = row;
              else if (P.pos[row] < P.pos[col]) target = up_blk(row, col);
              else target = lo_blk(col, row);
              const int tors = s_jl_law[jl0 + q] == LAW_TORSIONAL ? exg_newton::kTermTorsional : 0;
              cells[target].push_back((q * 4 + re * 2 + ce) | tors);
            }
          }
        }
        int pos = base_cell_terms + (int)s_cell_terms.size();
        for (int t = 0; t < n_cells; ++t) {
          s_cell_ptr.push_back(pos);
          for (int x : cells[t]) { s_cell_terms.push_back(x); ++pos; }
        }
        s_cell_ptr.push_back(pos);
      }
      desc.push_back(d);
      lens.push_back((scratch_doubles(d.nb, d.nj, m, d.n_slots) + 31) & ~31LL);
      continue;
    }
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
            // term: joint * 4 + row end * 2 + column end, bit kTermTorsional for the torsional law
            const int tors = s_jl_law[jl0 + q] == LAW_TORSIONAL ? exg_newton::kTermTorsional : 0;
            cells[target].push_back((q * 4 + re * 2 + ce) | tors);
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
  // one-writer ledger over the maps just built (crates/newton/src/accelerator/shaders.rs:321-390):
  // each body in one island, each joint end gathered once, each assembly term in one cell, each
  // factor block the target of one update group; a clash refuses the world before anything changes
  {
    std::vector<int32_t> v;
    for (int x : s_isl_body) v.push_back(x - body_off);
    int rc = exg_internal_ledger(v.data(), (long long)v.size(), n, nullptr, "structure refused: island bodies");
    for (size_t I = 0; I < desc.size() && rc == EXG_OK; ++I) {
      const IslandDesc& d = desc[I];
      const int li = d.inc_off - base_inc_ptr;
      const int r0 = s_ib_inc_ptr[li] - base_inc_ref, r1 = s_ib_inc_ptr[li + d.nb] - base_inc_ref;
      if (r1 - r0 != 2 * d.nj) {
        exg_internal_set_message("structure refused: an island gathers a joint end twice or not at all");
        rc = EXG_ERR_BACKEND;
      }
      if (rc == EXG_OK)
        rc = exg_internal_ledger(s_ib_inc_ref.data() + r0, r1 - r0, 2LL * d.nj, nullptr,
                                 "structure refused: gathered joint ends");
      const int lc = d.cell_off - base_cell_ptr;
      const int n_cells = d.solver == 1 ? d.m + 2 * d.n_slots : 3 * d.m;
      const int t0 = s_cell_ptr[lc] - base_cell_terms, t1 = s_cell_ptr[lc + n_cells] - base_cell_terms;
      v.assign(s_cell_terms.begin() + t0, s_cell_terms.begin() + t1);
      for (int32_t& x : v) x &= ~exg_newton::kTermTorsional;
      if (rc == EXG_OK) rc = exg_internal_ledger(v.data(), (long long)v.size(), 4LL * d.nj, nullptr,
                                                 "structure refused: assembly terms");
      if (rc == EXG_OK && d.solver == 1) {
        const int lg = d.gen_lv_off - base_gn_lgrp;
        const int g0 = s_gn_lgrp[lg] - base_gn_grp, g1 = s_gn_lgrp[lg + d.n_levels] - base_gn_grp;
        v.clear();
        for (int g = g0; g < g1; ++g) v.push_back(s_gn_grp[g].x);
        rc = exg_internal_ledger(v.data(), (long long)v.size(), (long long)d.m + 2LL * d.n_slots, nullptr,
                                 "structure refused: factor update targets");
      }
    }
    if (rc != EXG_OK) return rc;
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
  cat(h_jl_id, s_jl_id);
  cat(h_gn_lgrp, s_gn_lgrp); cat(h_gn_rop_ptr, s_gn_rop_ptr); cat(h_gn_slot_ptr, s_gn_slot_ptr);
  cat(h_gn_slot_col, s_gn_slot_col);
  h_gn_grp.insert(h_gn_grp.end(), s_gn_grp.begin(), s_gn_grp.end());
  h_gn_ops.insert(h_gn_ops.end(), s_gn_ops.begin(), s_gn_ops.end());
  h_gn_rops.insert(h_gn_rops.end(), s_gn_rops.begin(), s_gn_rops.end());
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

bool NewtonWorld::kin_differs(int slot, const exg_body_t* bodies, int n) const {
  if (slot < 0 || slot >= (int)src_.size() || !src_[slot].live) return false;
  const std::vector<char>& k = src_[slot].kin;
  if ((int)k.size() != n) return true;
  for (int i = 0; i < n; ++i)
    if (k[i] != (bodies[i].kinematic != 0)) return true;
  return false;
}

std::vector<char> NewtonWorld::kin_of(int slot) const {
  if (slot < 0 || slot >= (int)src_.size() || !src_[slot].live) return {};
  return src_[slot].kin;
}

int NewtonWorld::rebuild_from(int slot, WorldSrc next) {
  WorldSrc old = src_[slot];
  remove_world(slot);
  int rc = build_world(slot, next);
  if (rc != EXG_OK) {
    if (build_world(slot, old) == EXG_OK) src_[slot] = old;  // accepted before
    return rc;
  }
  next.live = true;
  src_[slot] = std::move(next);
  return EXG_OK;
}

int NewtonWorld::rebuild_world(int slot, const std::vector<char>& kin) {
  if (slot < 0 || slot >= (int)src_.size() || !src_[slot].live || src_[slot].kin.size() != kin.size())
    return EXG_ERR_INVALID_ARGUMENT;
  WorldSrc next = src_[slot];
  next.kin = kin;
  return rebuild_from(slot, std::move(next));
}

int NewtonWorld::replace_joints(int slot, const exg_joint_t* joints, int nj) {
  if (slot < 0 || slot >= (int)src_.size() || !src_[slot].live || nj < 0) return EXG_ERR_INVALID_ARGUMENT;
  WorldSrc next = src_[slot];
  next.joints.assign(joints, joints + nj);
  return rebuild_from(slot, std::move(next));
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
  up(d_gn_lgrp, h_gn_lgrp); up(d_gn_rop_ptr, h_gn_rop_ptr); up(d_gn_slot_ptr, h_gn_slot_ptr);
  up(d_gn_slot_col, h_gn_slot_col); up(d_gn_grp, h_gn_grp); up(d_gn_ops, h_gn_ops); up(d_gn_rops, h_gn_rops);
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
  // queue of the island kernel's live islands, largest first, then the scheduler's counter
  std::vector<int> q;
  for (int I = 0; I < (int)desc_.size(); ++I) if (alive_[I] && !wave_island(desc_[I])) q.push_back(I);
  n_cta_ = (int)q.size();
  std::stable_sort(q.begin(), q.end(),
                   [&](int a, int b) { return desc_[a].nb + desc_[a].nj > desc_[b].nb + desc_[b].nj; });
  q.push_back(0);
  if ((rc = d_queue.assign(q.data(), (long long)q.size(), s)) != EXG_OK) return rc;
  arr = NewtonDeviceArrays{d_desc.ptr,      d_isl_body.ptr, d_jl_law.ptr,   d_jl_a.ptr,      d_jl_b.ptr,     d_jl_params.ptr,
                           d_ib_order.ptr,  d_ib_inc_ptr.ptr, d_ib_inc_ref.ptr, d_dn_body.ptr, d_dn_parent.ptr, d_lv_ptr.ptr,
                           d_lv_nodes.ptr,  d_ch_ptr.ptr,   d_ch_idx.ptr,   d_cell_ptr.ptr,  d_cell_terms.ptr,
                           d_gn_lgrp.ptr,   d_gn_grp.ptr,   d_gn_ops.ptr,   d_gn_rop_ptr.ptr, d_gn_rops.ptr,
                           d_gn_slot_ptr.ptr, d_gn_slot_col.ptr, d_scratch.ptr,
                           d_stats.ptr,     d_residual.ptr, d_phase.ptr};
  if ((rc = build_wave(s)) != EXG_OK) return rc;
  dirty_ = false;
  return EXG_OK;
}

int NewtonWorld::enqueue(exg_device_s* dev, DeviceWorld& w, cudaStream_t s) {
  if (n_cta_ == 0) return EXG_OK;
  if (dirty_) return EXG_ERR_INVALID_ARGUMENT;  // sync() first
  WorldRef W{w.pose,    w.mom,    w.mass,   w.inertia, w.kinematic,  w.diagonal, w.pos_mass,
             w.grav_partial, w.wparams, w.w_poff, w.w_splits, w.w_n, w.w_body_off, w.w_active, w.n};
  int* head = d_queue.ptr + n_cta_;
  // persistent CTAs: as many as can be resident at once
  // variant 0 FP64, 1 mixed, 2 mixed with Newton-Schulz pivots (some world asks for them)
  static int resident[3] = {0, 0, 0};
  const int mixed = w.precision != EXG_PRECISION_F64;
  bool ns = false;
  if (mixed)
    for (const exg_step_params_t& p : w.h_params) ns = ns || (p.newton_flags & EXG_NEWTON_NS_PIVOT) != 0;
  const int var = mixed ? (ns ? 2 : 1) : 0;
  if (resident[var] == 0) {
    int per_sm = 0;
    cudaError_t e =
        var == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_newton_step<true, true>, kThreads, 0)
        : var == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_newton_step<true, false>, kThreads, 0)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_newton_step<false, false>, kThreads, 0);
    resident[var] = (e == cudaSuccess && per_sm > 0) ? per_sm : 1;
  }
  int grid = std::min(n_cta_, std::max(1, dev->sm_count) * resident[var]);
  EXG_CUDA_TRY(cudaMemsetAsync(head, 0, sizeof(int), s));
  int tok = prof_begin(dev, PROF_NEWTON, s);
  if (var == 2)
    k_newton_step<true, true><<<grid, kThreads, 0, s>>>(arr, W, d_queue.ptr, n_cta_, head);
  else if (var == 1)
    k_newton_step<true, false><<<grid, kThreads, 0, s>>>(arr, W, d_queue.ptr, n_cta_, head);
  else
    k_newton_step<false, false><<<grid, kThreads, 0, s>>>(arr, W, d_queue.ptr, n_cta_, head);
  prof_end(dev, tok, s);
  return exg_after_launch(dev);
}

int NewtonWorld::island_count(int slot) const {
  if (slot < 0 || slot >= (int)world_islands_.size()) return 0;
  return (int)world_islands_[slot].size();
}

int NewtonWorld::read_structure(int slot, int k, int kind, int* out, int cap, int* len) {
  if (dirty_) return EXG_ERR_INVALID_ARGUMENT;
  if (slot < 0 || slot >= (int)world_islands_.size() || k < 0 || k >= (int)world_islands_[slot].size())
    return EXG_ERR_INVALID_ARGUMENT;
  const IslandDesc& d = desc_[world_islands_[slot][k]];
  std::vector<int> v;
  cudaError_t err = cudaSuccess;
  auto fetch = [&](const DevArr<int>& a, long long off, int n) {
    std::vector<int> h(std::max(n, 0), 0);
    if (n > 0 && err == cudaSuccess) err = cudaMemcpy(h.data(), a.ptr + off, sizeof(int) * n, cudaMemcpyDeviceToHost);
    return h;
  };
  switch (kind) {
    case EXG_STRUCT_ISLAND_BODIES:
      v = fetch(d_isl_body, d.body_off, d.nb);
      for (int& x : v) x -= src_[slot].body_off;
      break;
    case EXG_STRUCT_JOINT_ENDS: {
      std::vector<int> law = fetch(d_jl_law, d.joint_off, d.nj), a = fetch(d_jl_a, d.joint_off, d.nj),
                       b = fetch(d_jl_b, d.joint_off, d.nj);
      for (int q = 0; q < d.nj; ++q) { v.push_back(law[q]); v.push_back(a[q]); v.push_back(b[q]); }
      break;
    }
    case EXG_STRUCT_ORDER: v = fetch(d_ib_order, d.body_off, d.nb); break;
    case EXG_STRUCT_INCIDENCE_PTR: {
      v = fetch(d_ib_inc_ptr, d.inc_off, d.nb + 1);
      const int base = v.empty() ? 0 : v[0];
      for (int& x : v) x -= base;
      break;
    }
    case EXG_STRUCT_INCIDENCE: {
      std::vector<int> p = fetch(d_ib_inc_ptr, d.inc_off, d.nb + 1);
      v = fetch(d_ib_inc_ref, p.front(), p.back() - p.front());
      break;
    }
    case EXG_STRUCT_PARENT: v = fetch(d_dn_parent, d.dyn_off, d.m); break;
    case EXG_STRUCT_ISLAND_JOINTS: v.assign(h_jl_id.begin() + d.joint_off, h_jl_id.begin() + d.joint_off + d.nj); break;
    default: return EXG_ERR_INVALID_ARGUMENT;
  }
  EXG_CUDA_TRY(err);
  *len = (int)v.size();
  if ((int)v.size() > cap) return EXG_ERR_INVALID_ARGUMENT;
  if (!v.empty()) std::copy(v.begin(), v.end(), out);
  return EXG_OK;
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
