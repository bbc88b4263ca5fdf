// Wave schedule of the device Newton step for large islands.
//
// The island kernel (newton.cu) gives every island one CTA, which leaves a large island's
// thousands of bodies to 256 threads while the rest of the GPU may sit idle. The wave schedule
// runs the same step with every phase as a grid-wide kernel over the items of ALL large islands
// at once, and keeps each island's control flow — the span budget loop of Newton::solve_step
// (crates/newton/src/integrator/implicit/newton.rs:543-683), the Newton iterations and the
// backtracking line search of newton_solve (:334-530) — as a per-island state machine that small
// control kernels advance between the data phases. One "round" evaluates every island once (a
// Newton iterate or a line-search probe) and, where the island needs it, assembles and solves for
// a new direction or ends its span; rounds repeat until every island has finished the step.
//
// The per-item arithmetic is the island kernel's (newton_ops.cuh), and every reduction over an
// island's items runs in a fixed order (maxima through order-independent integer atomics, sums
// warp-strided in index order), so a world's result does not depend on the other islands in the
// wave. A round is one CUDA graph, captured once per structural change.
#include <algorithm>
#include <cstring>
#include <vector>
#include "newton_ops.cuh"

namespace {

using namespace exg_newton;

enum WaveState { WS_START = 0, WS_ITER = 1, WS_PROBE = 2, WS_DIR = 3, WS_END = 4, WS_DONE = 5 };
enum WaveEval { EV_NONE = 0, EV_FULL = 1, EV_JAC = 2, EV_PLAIN = 3 };
enum WaveFlag {
  F_START = 1,       // load the world state, best = vm
  F_COPY_BEST = 2,   // best = vm
  F_ACCEPT = 8,      // vm = trial
  F_BASE = 16,       // base = vm
  F_TRIAL = 32,      // trial = base + alpha dv
  F_COMMIT = 64,     // commit the span
};

struct WaveCtl {
  unsigned long long remaining;  // span budget units left (of 2^kMaxDepth)
  unsigned long long worst_bits; // max of the round's node residuals (non-negative doubles order as integers)
  double span, half, pf, vf, best, rnorm, carried_norm, alpha, a_norm2, massn, last_best;
  int state, eval, flags, depth;
  int spans, iters, maxdepth, it;
  int carried, lane, converged, assembled;
  int nz, singular, commit_converged, active;
  int mflip;  // 1: the scratch's mass and mass0 blocks trade places (see wave_ctx)
  int ns;     // Newton-Schulz pivot inverses (mixed path, EXG_NEWTON_NS_PIVOT)
  int warm;   // a solve of this step has filled every node's Dinv slot
  double frame[kFrameDoubles];  // the island's frame for this step (frame_make)
};

struct WaveArgs {
  NewtonDeviceArrays A;
  WorldRef W;
  WaveCtl* ctl;
  const int* isl;       // wave slot -> island
  const IslandDesc* wdesc;  // wave slot -> the island's descriptor (a copy, one load less)
  int n_isl;
  const int2* body;     // (slot, island body)
  int n_body;
  const int2* dyn;      // (slot, dynamic node)
  int n_dyn;
  const int2* joint;    // (slot, island joint)
  int n_joint;
  const int2* cell;     // (slot, assembly cell)
  const int2* cell_range;  // per cell item: [p0, p1) of its terms in A.cell_terms
  int n_cell;
  const int2* level;    // (slot, node) grouped by elimination level
  const int* dyn_first; // first dynamic-node item of each wave slot (n_isl + 1 entries)
  double* nodesq;       // per dynamic-node item: a sum of squares to reduce per island
  int* live;            // counters, see kLive* below
  // Item ranges (kRange* below; the joint items of each law and the nodes of each elimination
  // level are ranges of their own). Within a range items are ordered by slot, so slot k's items
  // are [seg[k], seg[k + 1]) of it: seg holds n_isl + 1 offsets per range.
  const int* seg;
  int n_ranges;
  int* act;             // this round's unfinished slots, ascending (k_w_round_items)
  int* pre;             // per range, n_isl + 1 entries: item offsets of the listed slots
};

// Ranges of WaveArgs::seg: the body, dynamic-node and cell items, then the joint items of law
// 0 .. 4 (4: the traced laws), then the nodes of elimination level 0, 1, ...
enum { kRangeBody = 0, kRangeDyn = 1, kRangeCell = 2, kRangeJoint = 3, kRangeLevel = 8 };

int grid_for(exg_device_s* dev, long long items, int threads, int per_sm) {
  long long g = (items + threads - 1) / threads;
  long long cap = (long long)std::max(1, dev->sm_count) * per_sm;
  return (int)std::max<long long>(1, std::min(g, cap));
}

// Device counters of the wave (a.live): islands still stepping after the last round, rounds of
// this step, the round cap reached with islands unfinished, and cumulative rounds / direction
// sections / end sections (for the host's count of launched kernels).
// kLiveListed / kLiveSparse: the slots k_w_round_items listed for this round and whether the
// data kernels walk only their items.
enum { kLiveIslands = 0, kLiveRounds = 1, kLiveOverflow = 2, kLiveTotalRounds = 3, kLiveTotalDir = 4,
       kLiveTotalEnd = 5, kLiveListed = 6, kLiveSparse = 7, kLiveCount = 8 };
// Rounds one step may take before the wave gives up on it (EXG_ERR_FATAL); a step of a
// well-formed island needs at most spans x iterations x (1 + probes), far fewer in practice.
constexpr int kMaxRoundsPerStep = 1 << 17;

__device__ __forceinline__ int gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int gthreads() { return gridDim.x * blockDim.x; }

// An island's context in the wave. "mass0 = mass" (the island kernel copies 36 values per node)
// is a swap of the two block arrays' roles here: the evaluation writes the blocks into `mass`, and
// adopting them as mass0 flips mflip, so the next evaluation writes into the other array.
__device__ __forceinline__ Ctx wave_ctx(const WaveArgs& a, int k) {
  Ctx c = make_ctx_desc(a.A, a.W, a.wdesc[k], true);
  if (a.ctl[k].mflip) { double* t = c.s.mass; c.s.mass = c.s.mass0; c.s.mass0 = t; }
  c.frame = a.ctl[k].frame;
  return c;
}
__device__ __forceinline__ Ctx wave_ctx_lite(const WaveArgs& a, int k) {
  Ctx c = make_ctx_desc(a.A, a.W, a.wdesc[k], false);
  if (a.ctl[k].mflip) { double* t = c.s.mass; c.s.mass = c.s.mass0; c.s.mass0 = t; }
  return c;
}

// ── per-island control ──────────────────────────────────────────────────────
// Step start: every island of an active world begins its span budget; load the external wrench.
__global__ void k_w_init(WaveArgs a) {
  if (gtid() == 0) {
    a.live[kLiveRounds] = 0;
    a.live[kLiveOverflow] = 0;
    a.live[kLiveSparse] = 0;
  }
  for (int k = gtid(); k < a.n_isl; k += gthreads()) {
    WaveCtl& c = a.ctl[k];
    const IslandDesc& d = a.wdesc[k];
    c.active = a.W.w_active[d.world];
    c.state = c.active ? WS_START : WS_DONE;
    c.remaining = 1ull << kMaxDepth;
    c.depth = 0;
    c.spans = c.iters = c.maxdepth = 0;
    c.last_best = 0.0;
    c.flags = 0;
    c.eval = EV_NONE;
    c.mflip = 0;
    c.ns = (a.W.wparams[d.world].newton_flags & EXG_NEWTON_NS_PIVOT) != 0;
    c.warm = 0;
  }
}

// Step start, after k_w_init: every active island's frame for the step (its centre of mass), one
// CTA per island, the island kernel's arithmetic.
__global__ void __launch_bounds__(kFrameThreads) k_w_frame(WaveArgs a) {
  __shared__ double sh[4 * kFrameThreads];
  for (int k = blockIdx.x; k < a.n_isl; k += gridDim.x) {
    if (!a.ctl[k].active) continue;  // uniform over the CTA
    island_frame(a.A, a.W, a.wdesc[k], sh, a.ctl[k].frame);
  }
}

__global__ void k_w_external(WaveArgs a) {
  for (int t = gtid(); t < a.n_body; t += gthreads()) {
    int2 it = a.body[t];
    if (!a.ctl[it.x].active) continue;
    Ctx c = wave_ctx(a, it.x);
    op_load_external(c, it.y);
  }
}

// Round start: islands starting a span choose its length (the top of solve_step's budget loop);
// islands at an iterate or a probe choose what to evaluate.
__global__ void k_w_begin(WaveArgs a) {
  for (int k = gtid(); k < a.n_isl; k += gthreads()) {
    WaveCtl& c = a.ctl[k];
    c.flags = 0;
    c.eval = EV_NONE;
    c.worst_bits = 0ull;
    if (c.state == WS_START) {
      unsigned long long units = 1ull << (kMaxDepth - c.depth);
      while (units > c.remaining) { ++c.depth; units >>= 1; }
      const IslandDesc& d = a.wdesc[k];
      double span = a.W.wparams[d.world].dt;
      for (int t = 0; t < c.depth; ++t) span = span / 2.0;
      c.span = span;
      c.half = span / 2.0;
      const double scale = (a.W.wparams[d.world].newton_flags & EXG_NEWTON_EXACT_POSE_FACTOR) ? 0.5 : 1.0;
      c.pf = -(c.half * c.half) * scale;
      c.vf = -c.half;
      ++c.spans;
      c.maxdepth = max(c.maxdepth, c.depth);
      c.best = kHuge;
      c.converged = 0;
      c.assembled = 0;
      c.a_norm2 = 0.0;
      c.carried = 0;
      c.it = 0;
      c.flags = F_START;
      c.state = WS_ITER;
    }
    if (c.state == WS_ITER) {
      const IslandDesc& d = a.wdesc[k];
      const exg_step_params_t& wp = a.W.wparams[d.world];
      const int max_newton = wp.max_newton > 0 ? wp.max_newton : 32;
      if (c.it >= max_newton) {
        c.state = WS_END;
      } else {
        ++c.iters;
        c.eval = c.carried ? EV_JAC : EV_FULL;
      }
    } else if (c.state == WS_PROBE) {
      c.eval = EV_PLAIN;
    }
  }
}

// After the evaluation: the iterate's convergence test or the probe's acceptance test.
__global__ void k_w_after_eval(WaveArgs a) {
  for (int k = gtid(); k < a.n_isl; k += gthreads()) {
    WaveCtl& c = a.ctl[k];
    if (c.eval == EV_FULL || c.eval == EV_JAC) {
      const IslandDesc& d = a.wdesc[k];
      const exg_step_params_t& wp = a.W.wparams[d.world];
      double rnorm;
      if (c.eval == EV_JAC) {
        rnorm = c.carried_norm;
      } else {
        rnorm = __longlong_as_double((long long)c.worst_bits);
        c.mflip ^= 1;  // mass0 = mass
      }
      c.carried = 0;
      c.rnorm = rnorm;
      if (rnorm < c.best) {
        c.best = rnorm;
        c.flags |= F_COPY_BEST;
      }
      if (rnorm <= wp.tol * wp.tol) {
        c.converged = 1;
        c.state = WS_END;
      } else if (!(rnorm < kHuge)) {
        c.state = WS_END;
      } else {
        c.state = WS_DIR;
        c.nz = 0;
        c.singular = 0;
      }
    } else if (c.eval == EV_PLAIN) {
      const IslandDesc& d = a.wdesc[k];
      const exg_step_params_t& wp = a.W.wparams[d.world];
      const int max_newton = wp.max_newton > 0 ? wp.max_newton : 32;
      double tnorm = __longlong_as_double((long long)c.worst_bits);
      bool acc = tnorm < c.rnorm;
      if (c.lane == 0 || acc) c.mflip ^= 1;  // mass0 = mass
      if (acc) {
        c.flags |= F_ACCEPT;
        c.carried = 1;
        c.carried_norm = tnorm;
        ++c.it;
        c.state = c.it < max_newton ? WS_ITER : WS_END;
      } else {
        c.alpha = c.alpha / 2.0;
        ++c.lane;
        if (c.lane < kLineSearchLanes) c.flags |= F_TRIAL;
        else c.state = WS_END;  // no probe decreased the residual: vm still holds the base
      }
    }
  }
}

// After the solve: no correction at all hands over to sub-division (newton.rs:449-456);
// otherwise the line search starts at alpha = 1.
__global__ void k_w_after_solve(WaveArgs a) {
  for (int k = gtid(); k < a.n_isl; k += gthreads()) {
    WaveCtl& c = a.ctl[k];
    c.flags &= ~(F_COPY_BEST | F_ACCEPT | F_TRIAL);  // done by the post-evaluation copy pass
    if (c.state != WS_DIR) continue;
    c.assembled = 1;
    c.warm = 1;
    if (!c.nz) {
      c.state = WS_END;
      continue;
    }
    c.flags |= F_BASE | F_TRIAL;
    c.lane = 0;
    c.alpha = 1.0;
    c.state = WS_PROBE;
  }
}

// End of a span (the bottom of solve_step's budget loop): sub-divide, or commit and move on.
__global__ void k_w_end(WaveArgs a) {
  for (int k = gtid(); k < a.n_isl; k += gthreads()) {
    WaveCtl& c = a.ctl[k];
    c.flags &= ~(F_BASE | F_TRIAL);
    if (c.state != WS_END) continue;
    c.last_best = c.best;
    const bool finite = c.best < kHuge;
    const bool last = c.depth == kMaxDepth;
    int r;
    const bool sig = signal_from_norms(c.assembled != 0, c.a_norm2, c.massn, &r);
    if (!c.converged && !last) {
      int down = sig ? div_euclid(r - kThresholdLog2, kPerHalvingLog2) + 1 : 1;
      c.depth += min(max(down, 1), kMaxDepth - c.depth);
      c.state = WS_START;
      continue;
    }
    if (c.converged || finite) {
      c.flags |= F_COMMIT;
      c.commit_converged = c.converged;
    }
    unsigned long long units = 1ull << (kMaxDepth - c.depth);
    c.remaining -= units;
    auto aligned = [&](int dd) {
      if (dd <= 0) return false;
      unsigned long long bigger = 1ull << (kMaxDepth - (dd - 1));
      return bigger <= c.remaining && c.remaining % bigger == 0;
    };
    if (c.remaining > 0 && c.converged && aligned(c.depth) && sig) {
      int up = div_euclid(kThresholdLog2 - r, kPerHalvingLog2);
      while (up > 0 && aligned(c.depth)) { --c.depth; --up; }
    }
    if (c.remaining > 0) {
      c.state = WS_START;
    } else {
      c.state = WS_DONE;
      const int island = a.isl[k];
      a.A.stats[4 * island + 0] = c.spans;
      a.A.stats[4 * island + 1] = c.iters;
      a.A.stats[4 * island + 2] = c.maxdepth;
      a.A.stats[4 * island + 3] = (c.last_best < kHuge) ? 0 : 1;
      a.A.residual[island] = c.last_best;
    }
  }
}

// Whether any island is in `state` after the previous kernels: the condition of the round's
// direction (WS_DIR) or span-end (WS_END) section. One block.
__global__ void k_w_cond(WaveArgs a, cudaGraphConditionalHandle h, int state, int counter) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  int mine = 0;
  for (int k = threadIdx.x; k < a.n_isl; k += blockDim.x) mine |= a.ctl[k].state == state;
  if (mine) atomicOr(&any, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (any) atomicAdd(&a.live[counter], 1);
    cudaGraphSetConditional(h, any ? 1u : 0u);
  }
}

// Round end: islands still stepping; the loop's condition (some island unfinished and the cap not
// reached). One block.
__global__ void k_w_count(WaveArgs a, cudaGraphConditionalHandle h_loop) {
  __shared__ int n;
  if (threadIdx.x == 0) n = 0;
  __syncthreads();
  int mine = 0;
  for (int k = threadIdx.x; k < a.n_isl; k += blockDim.x) mine += a.ctl[k].state != WS_DONE;
  atomicAdd(&n, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    a.live[kLiveIslands] = n;
    const int r = ++a.live[kLiveRounds];
    ++a.live[kLiveTotalRounds];
    const bool over = n > 0 && r >= kMaxRoundsPerStep;
    if (over) a.live[kLiveOverflow] = 1;
    cudaGraphSetConditional(h_loop, (n > 0 && !over) ? 1u : 0u);
  }
}

// Round end of the host-driven form: islands still stepping, the round counters. One block.
__global__ void k_w_count_flat(WaveArgs a) {
  __shared__ int n;
  if (threadIdx.x == 0) n = 0;
  __syncthreads();
  int mine = 0;
  for (int k = threadIdx.x; k < a.n_isl; k += blockDim.x) mine += a.ctl[k].state != WS_DONE;
  atomicAdd(&n, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    a.live[kLiveIslands] = n;
    ++a.live[kLiveRounds];
  }
}

// Round start: the slots still stepping (state other than WS_DONE, which no island leaves before
// the step ends), ascending. When they are at most a sixteenth of all slots (a step's last rounds,
// where a few islands iterate or sub-divide on after the rest have committed) the round is sparse:
// for every range, one warp sums the listed slots' item counts into pre, and the data kernels walk
// those items only (RoundItems). With more slots listed, the search that maps an item number to
// its item costs more than skipping the finished islands' items. One block.
constexpr int kListThreads = 1024;
__global__ void __launch_bounds__(kListThreads) k_w_round_items(WaveArgs a) {
  __shared__ int warp_sum[kListThreads / 32];
  __shared__ int listed;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) listed = 0;
  __syncthreads();
  for (int k0 = 0; k0 < a.n_isl; k0 += kListThreads) {
    const int k = k0 + threadIdx.x;
    const int on = (k < a.n_isl && a.ctl[k].state != WS_DONE) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, on);
    if (lane == 0) warp_sum[wid] = __popc(bal);
    __syncthreads();
    int before = listed;
    for (int u = 0; u < wid; ++u) before += warp_sum[u];
    if (on) a.act[before + __popc(bal & ((1u << lane) - 1u))] = k;
    __syncthreads();
    if (threadIdx.x == kListThreads - 1) listed = before + __popc(bal);
    __syncthreads();
  }
  const int n_act = listed;
  const int sparse = 16 * n_act <= a.n_isl ? 1 : 0;
  if (threadIdx.x == 0) {
    a.live[kLiveListed] = n_act;
    a.live[kLiveSparse] = sparse;
  }
  if (!sparse) return;
  const int stride = a.n_isl + 1;
  for (int r = wid; r < a.n_ranges; r += kListThreads / 32) {
    const int* sg = a.seg + (size_t)r * stride;
    int* pr = a.pre + (size_t)r * stride;
    if (lane == 0) pr[0] = 0;
    int carry = 0;
    for (int i0 = 0; i0 < n_act; i0 += 32) {
      const int i = i0 + lane;
      int c = 0;
      if (i < n_act) {
        const int k = a.act[i];
        c = sg[k + 1] - sg[k];
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, c, o);
        if (lane >= o) c += y;
      }
      if (i < n_act) pr[i + 1] = carry + c;
      carry += __shfl_sync(0xffffffffu, c, 31);
    }
  }
}

// The items of one range that a data kernel visits this round, numbered 0 .. n-1: all of them, or
// in a sparse round those of the listed slots in slot order (at() maps the number to the item's
// offset in the range by a search of pre). Which items a kernel skips, and the arithmetic of those
// it does not, are the same in both forms.
struct RoundItems {
  int n;
  int n_act;
  const int* pre;  // nullptr: every item, at(v) = v
  const int* seg;
  const int* act;
  __device__ __forceinline__ int at(int v) const {
    if (!pre) return v;
    int lo = 0, hi = n_act - 1;  // the last listed slot whose items start at or before v
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (pre[mid] <= v) lo = mid;
      else hi = mid - 1;
    }
    return seg[act[lo]] + (v - pre[lo]);
  }
};

__device__ __forceinline__ RoundItems round_items(const WaveArgs& a, int range, int n) {
  RoundItems r;
  r.n = n;
  r.n_act = 0;
  r.pre = nullptr;
  r.seg = nullptr;
  r.act = nullptr;
  if (a.live[kLiveSparse]) {
    const size_t stride = (size_t)a.n_isl + 1;
    r.n_act = a.live[kLiveListed];
    r.pre = a.pre + range * stride;
    r.seg = a.seg + range * stride;
    r.act = a.act;
    r.n = r.pre[r.n_act];
  }
  return r;
}

// ── data phases over all islands' items ─────────────────────────────────────
__global__ void k_w_start(WaveArgs a) {
  const RoundItems R = round_items(a, kRangeBody, a.n_body);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.body[t];
    if (!(a.ctl[it.x].flags & F_START)) continue;
    Ctx c = wave_ctx(a, it.x);
    op_load_world_state(c, it.y);
    double v[6];
    ld_n<6>(c.s.vm + 6 * (size_t)it.y, v);
    st_n<6>(c.s.best + 6 * (size_t)it.y, v);
  }
}

__global__ void k_w_pre(WaveArgs a) {
  const RoundItems R = round_items(a, kRangeBody, a.n_body);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.body[t];
    const WaveCtl& w = a.ctl[it.x];
    if (w.eval != EV_FULL && w.eval != EV_PLAIN) continue;
    Ctx c = wave_ctx(a, it.x);
    op_pre(c, w.eval == EV_FULL ? c.s.vm : c.s.trial, w.half, it.y);
  }
}

// Joint tasks of one law (joint items are grouped by law; items [first, first + n) carry LAW),
// one instantiation per law and task kind so each keeps its own register budget:
//   slices: [0, 4 n) Jacobian slices, for an iterate (afresh or carried over from a probe);
//   values: [0, n) FP64 values, for an iterate evaluated afresh (mixed path; in FP64 the slices'
//           value parts are the values) and for a probe. A carried iterate keeps the values the
//           accepted probe left at the same point.
// A joint's four slices are evaluated as eight half slices (3 axes each: half the dual state per
// thread, so more threads fit on an SM), in two launches: KIND 0 the pose slices (0, 1), KIND 1 the
// twist slices (2, 3), whose laws run their pose chains without partials and so need far fewer
// registers. A warp takes 8 joints, four lanes each. Each lane writes its part of the slice
// records into the warp's staging block in shared memory, and the warp then stores each joint's
// two contiguous records (2 x 36 values, 16-byte aligned) with 16-byte stores.
template <bool MIXED, int LAW, int KIND>
__global__ void __launch_bounds__(128, KIND == 0 ? 4 : 8) k_w_joint_slices(WaveArgs a, int first, int n, int range) {
  typedef typename JacType<MIXED>::T J;
  constexpr int kHalf = 2 * kJacStride;  // values per joint and kind
  __shared__ __align__(16) J stage[4][8][kHalf];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const RoundItems R = round_items(a, range, n);
  const long long total = 32LL * ((R.n + 7) / 8);
  for (long long base = gtid() - lane; base < total; base += gthreads()) {  // warp-uniform loop
    const int jq = (int)(base >> 5) * 8 + (lane >> 2), slice = 2 * KIND + ((lane >> 1) & 1), half = lane & 1;
    bool on = false;
    int2 it = make_int2(0, 0);
    if (jq < R.n) {
      it = a.joint[first + R.at(jq)];
      const int ev = a.ctl[it.x].eval;
      if (ev == EV_FULL || ev == EV_JAC) {
        on = true;
        Ctx c = wave_ctx(a, it.x);
        op_joint_half_slice<MIXED, LAW, KIND>(c, c.s.vm, it.y, slice, half, ev == EV_FULL,
                                        &stage[wib][lane >> 2][(slice & 1) * kJacStride]);
      }
    }
    const unsigned active = __ballot_sync(0xffffffffu, on);
    __syncwarp();
    for (int j = 0; j < 8; ++j) {
      if (!((active >> (4 * j)) & 1u)) continue;  // no joint here, or its island did not evaluate slices
      const int2 jt = make_int2(__shfl_sync(0xffffffffu, it.x, 4 * j), __shfl_sync(0xffffffffu, it.y, 4 * j));
      const IslandDesc& d = a.wdesc[jt.x];
      J* dstj = reinterpret_cast<J*>(carve(a.A.scratch + d.scratch_off, d.nb, d.nj, d.m).jac) +
                (size_t)jt.y * 4 * kJacStride + KIND * kHalf;
      const float4* src = reinterpret_cast<const float4*>(&stage[wib][j][0]);
      float4* dst4 = reinterpret_cast<float4*>(dstj);
      constexpr int kVec = kHalf * (int)sizeof(J) / 16;
      for (int v = lane; v < kVec; v += 32) dst4[v] = src[v];
    }
    __syncwarp();
  }
}

template <bool MIXED, int LAW>
__global__ void __launch_bounds__(128) k_w_joint_values(WaveArgs a, int first, int n, int range) {
  const RoundItems R = round_items(a, range, n);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.joint[first + t];
    const int ev = a.ctl[it.x].eval;
    // (no torsional slices are evaluated, so in FP64 the torsional values come from here too)
    if (!(ev == EV_PLAIN || (ev == EV_FULL && (MIXED || LAW == LAW_TORSIONAL)))) continue;
    Ctx c = wave_ctx(a, it.x);
    op_joint_value<LAW>(c, ev == EV_PLAIN ? c.s.trial : c.s.vm, it.y);
  }
}

// The slices of one law on s, its values on sv (independent work: slices write the Jacobian
// records, values the joint wrenches).
template <bool MIXED, int LAW>
void launch_joints_of(exg_device_s* dev, const WaveArgs& a, int first, int n, int range, cudaStream_t s,
                      cudaStream_t sv) {
  const int per = 2 * dev->tune_wave_blocks_per_sm;
  if (LAW != LAW_TORSIONAL) {  // the assembly knows the torsional slices in closed form
    const int g = grid_for(dev, 32LL * ((n + 7) / 8), 128, per);
    k_w_joint_slices<MIXED, LAW, 0><<<g, 128, 0, s>>>(a, first, n, range);
    k_w_joint_slices<MIXED, LAW, 1><<<g, 128, 0, s>>>(a, first, n, range);
  }
  k_w_joint_values<MIXED, LAW><<<grid_for(dev, n, 128, per), 128, 0, sv>>>(a, first, n, range);
}

template <bool MIXED>
void launch_joints_by_law(exg_device_s* dev, const WaveArgs& a, const int* law_first, cudaStream_t s,
                          cudaStream_t sv) {
  for (int L = 0; L < 5; ++L) {
    const int first = law_first[L], n = law_first[L + 1] - first;
    if (n == 0) continue;
    const int r = kRangeJoint + L;
    if (L == 0) launch_joints_of<MIXED, 0>(dev, a, first, n, r, s, sv);
    else if (L == 1) launch_joints_of<MIXED, 1>(dev, a, first, n, r, s, sv);
    else if (L == 2) launch_joints_of<MIXED, 2>(dev, a, first, n, r, s, sv);
    else if (L == 3) launch_joints_of<MIXED, 3>(dev, a, first, n, r, s, sv);
    else launch_joints_of<MIXED, -1>(dev, a, first, n, r, s, sv);  // traced laws: the law read per joint
  }
}

__global__ void __launch_bounds__(256, 2) k_w_post(WaveArgs a) {
  const RoundItems R = round_items(a, kRangeDyn, a.n_dyn);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.dyn[t];
    WaveCtl& w = a.ctl[it.x];
    if (w.eval != EV_FULL && w.eval != EV_PLAIN) continue;
    Ctx c = wave_ctx(a, it.x);
    double worst = op_post(c, w.eval == EV_FULL ? c.s.vm : c.s.trial, w.half, it.y);
    // non-negative doubles (and NaN, which must win as nan_max makes it win) order as integers
    atomicMax(&w.worst_bits, (unsigned long long)__double_as_longlong(worst));
  }
}

// Body copies of the control decisions, in a fixed order per body.
__global__ void k_w_copy_bodies(WaveArgs a) {
  const RoundItems R = round_items(a, kRangeBody, a.n_body);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.body[t];
    const WaveCtl& w = a.ctl[it.x];
    const int f = w.flags;
    if (!(f & (F_COPY_BEST | F_ACCEPT | F_BASE | F_TRIAL))) continue;
    Ctx c = wave_ctx(a, it.x);
    const size_t o = 6 * (size_t)it.y;
    double v[6];
    ld_n<6>(c.s.vm + o, v);
    if (f & F_COPY_BEST) st_n<6>(c.s.best + o, v);
    if (f & F_ACCEPT) {
      ld_n<6>(c.s.trial + o, v);
      st_n<6>(c.s.vm + o, v);
    }
    if (f & F_BASE) st_n<6>(c.s.base + o, v);
    if (f & F_TRIAL) {  // op_trial for the body's six entries
      const int i = c.A.ib_order[c.d.body_off + it.y];
      double bs[6], tr[6];
      ld_n<6>(c.s.base + o, bs);
      if (i >= 0) {
        double d[6];
        ld_n<6>(c.s.dv + 6 * (size_t)i, d);
#pragma unroll
        for (int k = 0; k < 6; ++k) tr[k] = bs[k] + d[k] * w.alpha;
      } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) tr[k] = bs[k];
      }
      st_n<6>(c.s.trial + o, tr);
    }
  }
}


// Four entries of a 6x6 block from 16-byte aligned storage.
__device__ __forceinline__ void load4(const float* p, float o[4]) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = x.w;
}
__device__ __forceinline__ void load4(const double* p, double o[4]) {
  const double2 x = reinterpret_cast<const double2*>(p)[0], y = reinterpret_cast<const double2*>(p)[1];
  o[0] = x.x; o[1] = x.y; o[2] = y.x; o[3] = y.y;
}

// Entries e0 .. e0+3 of one assembly term's pose (p) and velocity (v) blocks in slice precision;
// returns whether the row end flips their sign. A torsional term has them in closed form
// (joint_jacobian_part, value for value): zero pose columns, g = -/+ c / warp^2 on the angular
// diagonal (entries 21, 28, 35) of the velocity columns.
template <bool MIXED>
__device__ __forceinline__ bool asm_term(const Ctx& c, int raw, int e0, typename JacType<MIXED>::T p[4],
                                         typename JacType<MIXED>::T v[4]) {
  typedef typename JacType<MIXED>::T J;
  const int term = raw & ~kTermTorsional;
  const int q = term >> 2, ce = term & 1;
  if (raw & kTermTorsional) {
    const double warp = c.W.wparams[c.d.world].warp;
    const J kk = -J(c.A.jl_params[10 * (size_t)(c.d.joint_off + q)] / (warp * warp));
    const J g = ce == 0 ? kk : -kk;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int e = e0 + m;
      p[m] = J(0);
      v[m] = (e >= 21 && e % 7 == 0) ? g : J(0);
    }
  } else {
    load4(jac_slice<MIXED>(c, q, ce) + e0, p);
    load4(jac_slice<MIXED>(c, q, 2 + ce) + e0, v);
  }
  return (term >> 1) & 1;
}

// acc += pf p + vf v entry by entry, in FP64, with the term's sign (as op_assemble adds a term).
template <typename J>
__device__ __forceinline__ void asm_add(double acc[4], double pf, double vf, bool re, const J p[4], const J v[4]) {
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    double pv = double(p[m]), vv = double(v[m]);
    if (re) { pv = -pv; vv = -vv; }
    acc[m] = acc[m] + pf * pv + vf * vv;
  }
}

// Assembly, three cells per warp: nine lanes per cell, lane l holding entries 4l .. 4l+3, so a
// term's block is one 16-byte load per lane (FP32 slices) and the output two. Every entry adds
// the mass block and then its terms in cell order, as op_assemble does. (Taking two terms at a
// time, or fewer CTAs per SM with more registers, measured slower.)
template <bool MIXED>
__global__ void __launch_bounds__(256, 4) k_w_assemble(WaveArgs a) {
  typedef typename JacType<MIXED>::T J;
  const int lane = threadIdx.x & 31, grp = lane / 9, e0 = 4 * (lane - 9 * grp);
  const RoundItems R = round_items(a, kRangeCell, a.n_cell);
  for (int t0 = 3 * (gtid() >> 5); t0 < R.n; t0 += 3 * (gthreads() >> 5)) {
    if (grp >= 3 || t0 + grp >= R.n) continue;
    const int t = R.at(t0 + grp);
    const int2 it = a.cell[t], range = a.cell_range[t];
    const WaveCtl& w = a.ctl[it.x];
    if (w.state != WS_DIR) continue;
    const Ctx c = wave_ctx_lite(a, it.x);
    const double pf = w.pf, vf = w.vf;
    const int cell = it.y, i = cell / 3, kind = cell % 3;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (kind == 0) load4(c.s.mass0 + 36 * (size_t)i + e0, acc);
    const int* terms = c.A.cell_terms;
    const int p0 = range.x, p1 = range.y;
    // the group's nine lanes fetch nine term indices at a time and pass them round by shuffle, so
    // a term's block loads wait on no index load of their own
    const unsigned gmask = 0x1ffu << (9 * grp);
    const int sub = e0 >> 2;
    int mine = 0;
    for (int k = p0; k < p1; ++k) {
      const int j = (k - p0) % 9;
      if (j == 0) mine = (k + sub < p1) ? terms[k + sub] : 0;
      J pa[4], va[4];
      const bool ra = asm_term<MIXED>(c, __shfl_sync(gmask, mine, 9 * grp + j), e0, pa, va);
      asm_add(acc, pf, vf, ra, pa, va);
    }
    double* dst = (kind == 0 ? c.s.D : (kind == 1 ? c.s.Acp : c.s.Apc)) + 36 * (size_t)i + e0;
    reinterpret_cast<double2*>(dst)[0] = make_double2(acc[0], acc[1]);
    reinterpret_cast<double2*>(dst)[1] = make_double2(acc[2], acc[3]);
  }
}

// The islands whose span end reads the stiffness signal (not converged, sub-division left, a matrix
// assembled in the span): only they sum ||A||_F^2 and ||M||_F^2, at span end, from the blocks of
// their last assembly (the elimination leaves D, A_cp and A_pc as assembled), the same values the
// island kernel sums after each assembly.
__device__ __forceinline__ bool wants_norms(const WaveCtl& w) {
  return w.state == WS_END && w.assembled && !w.converged && w.depth != kMaxDepth;
}

// Per dynamic node, a fixed-order sum of squares: of its assembled blocks (the diagonal, and the
// two parent couplings of a non-root node) for ||A||_F^2, or of its mass0 block for ||M||_F^2.
__global__ void k_w_node_sq(WaveArgs a, int mass) {
  const RoundItems R = round_items(a, kRangeDyn, a.n_dyn);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.dyn[t];
    const WaveCtl& w = a.ctl[it.x];
    if (!wants_norms(w)) continue;
    Ctx c = wave_ctx_lite(a, it.x);
    const size_t o = 36 * (size_t)it.y;
    double s = 0.0;
    auto add_sq = [&](const double* blk) {  // entries in order, read two at a time
      const double2* b2 = reinterpret_cast<const double2*>(blk + o);
#pragma unroll 6
      for (int e = 0; e < 18; ++e) {
        const double2 v = b2[e];
        s += v.x * v.x;
        s += v.y * v.y;
      }
    };
    if (mass) {
      add_sq(c.s.mass0);
    } else {
      add_sq(c.s.D);
      if (c.A.dn_parent[c.d.dyn_off + it.y] >= 0) {
        add_sq(c.s.Acp);
        add_sq(c.s.Apc);
      }
    }
    a.nodesq[t] = s;
  }
}

// One CTA per island: the sum of its node values, thread-strided in index order and then a
// fixed-shape tree, so the result does not depend on scheduling.
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) k_w_island_sum(WaveArgs a, int mass) {
  __shared__ double part[kSumThreads];
  for (int k = blockIdx.x; k < a.n_isl; k += gridDim.x) {
    const WaveCtl& w = a.ctl[k];
    if (!wants_norms(w)) continue;
    const int first = a.dyn_first[k], count = a.dyn_first[k + 1] - first;
    double s = 0.0;
    for (int t = threadIdx.x; t < count; t += kSumThreads) s += a.nodesq[first + t];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int h = kSumThreads / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      if (mass) a.ctl[k].massn = part[0];
      else a.ctl[k].a_norm2 = part[0];
    }
    __syncthreads();
  }
}

// Elimination, one thread per node of level L (leaves to roots), the node's blocks in registers:
// subtract the children's Schur terms, invert the pivot block, and for a non-root node form its own
// terms for the parent — S = Apc Dinv, then P = S Acp (kept in S's slot) and q = S b (kept in dv's
// slot until the back substitution writes dv) — so a parent only sums finished products; a root
// solves for dv. The arithmetic per entry is the island kernel's (newton_ops.cuh).
// With Newton-Schulz pivots (mixed path, EXG_NEWTON_NS_PIVOT) the pivot block passes through two
// columns of shared memory per thread (the block, then the previous and the new inverse: 72 doubles
// a thread, 36 KB for the 64-thread CTA), so the FP32 iteration and the FP64 correction hold only
// their own blocks in registers; Gauss-Jordan pivots stay in registers.
template <bool NS>
constexpr int down_threads() { return NS ? 64 : 128; }
template <bool MIXED, bool NS>
__global__ void __launch_bounds__(down_threads<MIXED && NS>(), (MIXED && NS) ? 6 : 3)
    k_w_solve_down(WaveArgs a, int first, int count, int range) {
  extern __shared__ double w_pivot[];
  const RoundItems R = round_items(a, range, count);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.level[first + t];
    WaveCtl& w = a.ctl[it.x];
    if (w.state != WS_DIR) continue;
    Ctx c = wave_ctx_lite(a, it.x);
    const int i = it.y;
    double D[36], b[6];
    ld_n<36>(c.s.D + 36 * (size_t)i, D);
    ld_n<6>(c.s.rhs + 6 * (size_t)i, b);
    const int* chp = c.A.ch_ptr + c.d.dyn_off;
    for (int u = chp[i]; u < chp[i + 1]; ++u) {
      const int ch = c.A.ch_idx[u];
      const double2* P = reinterpret_cast<const double2*>(c.s.S + 36 * (size_t)ch);
#pragma unroll
      for (int e = 0; e < 18; ++e) {
        const double2 x = P[e];
        D[2 * e] = D[2 * e] - x.x;
        D[2 * e + 1] = D[2 * e + 1] - x.y;
      }
      const double2* q = reinterpret_cast<const double2*>(c.s.dv + 6 * (size_t)ch);
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const double2 x = q[r];
        b[2 * r] = b[2 * r] - x.x;
        b[2 * r + 1] = b[2 * r + 1] - x.y;
      }
    }
    st_n<6>(c.s.bvec + 6 * (size_t)i, b);
    double Dinv[36];
    if (MIXED && NS && w.ns) {
      constexpr int T = down_threads<MIXED && NS>();
      double* col = w_pivot + threadIdx.x;
#pragma unroll
      for (int e = 0; e < 36; ++e) col[e * T] = D[e];
      {
        const bool warm = w.warm != 0;
        if (warm) {
          const double2* xp = reinterpret_cast<const double2*>(c.s.Dinv + 36 * (size_t)i);
#pragma unroll
          for (int e = 0; e < 18; ++e) {
            const double2 x = xp[e];
            col[(36 + 2 * e) * T] = x.x;
            col[(37 + 2 * e) * T] = x.y;
          }
        }
        if (!thread_ns_inverse6<T>(col, col + 36 * T, warm)) atomicOr(&w.singular, 1);
      }
#pragma unroll
      for (int e = 0; e < 36; ++e) Dinv[e] = col[(36 + e) * T];
    } else {
      if (!thread_inverse6(D, Dinv)) atomicOr(&w.singular, 1);
    }
    st_n<36>(c.s.Dinv + 36 * (size_t)i, Dinv);
    if (c.A.dn_parent[c.d.dyn_off + i] >= 0) {
      double dv[6];
      const double* Acp = c.s.Acp + 36 * (size_t)i;
      const double* Apc = c.s.Apc + 36 * (size_t)i;
      double2* P = reinterpret_cast<double2*>(c.s.S + 36 * (size_t)i);
#pragma unroll
      for (int r = 0; r < 6; ++r) {
        double ar[6], Sr[6], Pr[6];
        ld_n<6>(Apc + 6 * r, ar);
#pragma unroll
        for (int cc = 0; cc < 6; ++cc) {
          double v = 0.0;
#pragma unroll
          for (int k = 0; k < 6; ++k) v += ar[k] * Dinv[k * 6 + cc];
          Sr[cc] = v;
        }
        double q = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) q += Sr[k] * b[k];
        dv[r] = q;
        // row r of P = S Acp, each entry summed over k in order (rows of Acp as 16-byte loads)
#pragma unroll
        for (int cc = 0; cc < 6; ++cc) Pr[cc] = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          double ak[6];
          ld_n<6>(Acp + 6 * k, ak);
#pragma unroll
          for (int cc = 0; cc < 6; ++cc) Pr[cc] += Sr[k] * ak[cc];
        }
#pragma unroll
        for (int e = 0; e < 3; ++e) P[3 * r + e] = make_double2(Pr[2 * e], Pr[2 * e + 1]);
      }
      st_n<6>(c.s.dv + 6 * (size_t)i, dv);
    } else {
      double dv[6];
#pragma unroll
      for (int r = 0; r < 6; ++r) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) v += Dinv[r * 6 + k] * b[k];
        dv[r] = v;
      }
      st_n<6>(c.s.dv + 6 * (size_t)i, dv);
    }
  }
}

// The same elimination with one warp per node, for narrow levels, where one thread's dependent
// chain (loads, the 6x6 inverse, two products) would bound the level's time. Entry e of a block
// is lane e (lanes 0..3 also e + 32); the blocks pass through the warp's shared memory to the
// warp-cooperative operations, which do per entry exactly the single-thread arithmetic, so the two
// kernels give the same bits.
constexpr int kSolveWarps = 4;
// Levels of at most dev->tune_wave_narrow_level nodes (default 8192) take the warp kernel, wider
// ones the thread kernel; the autotuner measures the threshold.
// A narrow level is a chain of dependent loads per node; the kernel issues every load that waits
// on no other one together at the start (the node's blocks and right-hand side, the parent
// couplings staged into shared memory for the products, the children's range) and fetches the
// children's finished products four at a time, subtracting them in child order.
template <bool MIXED, bool NS>
__global__ void __launch_bounds__(32 * kSolveWarps) k_w_solve_down_warp(WaveArgs a, int first, int count, int range) {
  __shared__ __align__(16) double sh[kSolveWarps][36 * 5 + 8];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* Dm = sh[wib];
  double* Dinv = Dm + 36;
  double* S = Dm + 72;
  double* Ap = Dm + 108;  // A_pc, staged
  double* Ac = Dm + 144;  // A_cp, staged
  double* b = Dm + 180;
  const int e1 = lane + 32;
  const bool has1 = e1 < 36;
  const RoundItems R = round_items(a, range, count);
  for (int vi = gtid() >> 5; vi < R.n; vi += gthreads() >> 5) {  // warp-uniform
    const int t = R.at(vi);
    const int2 it = a.level[first + t];
    WaveCtl& w = a.ctl[it.x];
    if (w.state != WS_DIR) continue;
    const Ctx c = wave_ctx_lite(a, it.x);
    const size_t i = it.y;
    const int* chp = c.A.ch_ptr + c.d.dyn_off;
    const int u0 = chp[i], u1 = chp[i + 1];
    const int par = c.A.dn_parent[c.d.dyn_off + i];
    double d0 = c.s.D[36 * i + lane], d1 = has1 ? c.s.D[36 * i + e1] : 0.0;
    double bb = lane < 6 ? c.s.rhs[6 * i + lane] : 0.0;
    // a root's coupling slots hold nothing it reads; loading them anyway keeps the loads unconditional
    const double ap0 = c.s.Apc[36 * i + lane], ap1 = has1 ? c.s.Apc[36 * i + e1] : 0.0;
    const double ac0 = c.s.Acp[36 * i + lane], ac1 = has1 ? c.s.Acp[36 * i + e1] : 0.0;
    for (int ub = u0; ub < u1; ub += 32) {
      const int nc = min(32, u1 - ub);
      const int chl = lane < nc ? c.A.ch_idx[ub + lane] : 0;
      int k = 0;
      for (; k + 4 <= nc; k += 4) {
        size_t ch[4];
        double p0[4], p1[4], q[4];
#pragma unroll
        for (int h = 0; h < 4; ++h) ch[h] = (size_t)__shfl_sync(0xffffffffu, chl, k + h);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          p0[h] = c.s.S[36 * ch[h] + lane];
          p1[h] = has1 ? c.s.S[36 * ch[h] + e1] : 0.0;
          q[h] = lane < 6 ? c.s.dv[6 * ch[h] + lane] : 0.0;
        }
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          d0 = d0 - p0[h];
          if (has1) d1 = d1 - p1[h];
          if (lane < 6) bb = bb - q[h];
        }
      }
      for (; k < nc; ++k) {
        const size_t ch = (size_t)__shfl_sync(0xffffffffu, chl, k);
        d0 = d0 - c.s.S[36 * ch + lane];
        if (has1) d1 = d1 - c.s.S[36 * ch + e1];
        if (lane < 6) bb = bb - c.s.dv[6 * ch + lane];
      }
    }
    Dm[lane] = d0;
    Ap[lane] = ap0;
    Ac[lane] = ac0;
    if (has1) {
      Dm[e1] = d1;
      Ap[e1] = ap1;
      Ac[e1] = ac1;
    }
    if (lane < 6) {
      b[lane] = bb;
      c.s.bvec[6 * i + lane] = bb;
    }
    __syncwarp();
    if (MIXED && NS && w.ns && w.warm) {  // the node's inverse from the previous solve, the Newton-Schulz start
      Dinv[lane] = c.s.Dinv[36 * i + lane];
      if (has1) Dinv[e1] = c.s.Dinv[36 * i + e1];
      __syncwarp();
    }
    if (!warp_pivot_inverse6<MIXED && NS>(Dm, Dinv, w.ns != 0, w.warm != 0) && lane == 0) atomicOr(&w.singular, 1);
    c.s.Dinv[36 * i + lane] = Dinv[lane];
    if (has1) c.s.Dinv[36 * i + e1] = Dinv[e1];
    if (par >= 0) {
      warp_mm6<false>(Ap, Dinv, S);                   // S = Apc Dinv
      warp_mm6<false>(S, Ac, c.s.S + 36 * i);         // P = S Acp, in S's slot
      warp_mv6(S, b, c.s.dv + 6 * i);                 // q = S b, in dv's slot
    } else {
      warp_mv6(Dinv, b, c.s.dv + 6 * i);
    }
    __syncwarp();
  }
}

__global__ void k_w_solve_up(WaveArgs a, int first, int count, int range) {
  const RoundItems R = round_items(a, range, count);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.level[first + t];
    if (a.ctl[it.x].state != WS_DIR) continue;
    Ctx c = wave_ctx_lite(a, it.x);
    const int i = it.y;
    const int p = c.A.dn_parent[c.d.dyn_off + i];
    const double* Acp = c.s.Acp + 36 * (size_t)i;
    const double* Dinv = c.s.Dinv + 36 * (size_t)i;
    double xp[6], b[6], x[6];
    ld_n<6>(c.s.dv + 6 * (size_t)p, xp);
    ld_n<6>(c.s.bvec + 6 * (size_t)i, b);
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double ar[6];
      ld_n<6>(Acp + 6 * r, ar);
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) v += ar[k] * xp[k];
      b[r] = b[r] - v;
    }
    st_n<6>(c.s.bvec + 6 * (size_t)i, b);
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double dr[6];
      ld_n<6>(Dinv + 6 * r, dr);
      double v = 0.0;
#pragma unroll
      for (int k = 0; k < 6; ++k) v += dr[k] * b[k];
      x[r] = v;
    }
    st_n<6>(c.s.dv + 6 * (size_t)i, x);
  }
}

// Back substitution with one warp per node (lanes 0..5 one row each), for narrow levels: each lane
// loads its rows of A_cp and D^-1 and its right-hand side entry while the parent index resolves,
// then y = b - A_cp x_p and x = D^-1 y with y passed by shuffle; the same sums in the same order
// as warp_mv6_sub / warp_mv6.
__global__ void __launch_bounds__(32 * kSolveWarps) k_w_solve_up_warp(WaveArgs a, int first, int count, int range) {
  const int lane = threadIdx.x & 31;
  const RoundItems R = round_items(a, range, count);
  for (int vi = gtid() >> 5; vi < R.n; vi += gthreads() >> 5) {  // warp-uniform
    const int t = R.at(vi);
    const int2 it = a.level[first + t];
    if (a.ctl[it.x].state != WS_DIR) continue;
    const Ctx c = wave_ctx_lite(a, it.x);
    const size_t i = it.y;
    const size_t p = c.A.dn_parent[c.d.dyn_off + i];
    const int r = lane < 6 ? lane : 0;
    double ar[6], dr[6], xp[6];
    ld_n<6>(c.s.Acp + 36 * i + 6 * r, ar);
    ld_n<6>(c.s.Dinv + 36 * i + 6 * r, dr);
    double y = c.s.bvec[6 * i + r];
    ld_n<6>(c.s.dv + 6 * p, xp);
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) s += ar[k] * xp[k];
    y = y - s;
    if (lane < 6) c.s.bvec[6 * i + lane] = y;
    double x = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) x += dr[k] * __shfl_sync(0xffffffffu, y, k);
    if (lane < 6) c.s.dv[6 * i + lane] = x;
  }
}

// A singular pivot makes the whole correction NaN (the line search then rejects it); otherwise
// record whether any component is non-zero.
__global__ void k_w_nz(WaveArgs a) {
  const RoundItems R = round_items(a, kRangeDyn, a.n_dyn);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.dyn[t];
    WaveCtl& w = a.ctl[it.x];
    if (w.state != WS_DIR) continue;
    Ctx c = wave_ctx(a, it.x);
    double* dv = c.s.dv + 6 * (size_t)it.y;
    int nz = 0;
    if (w.singular) {
      const double nan = __longlong_as_double(0x7ff8000000000000LL);
      const double v[6] = {nan, nan, nan, nan, nan, nan};
      st_n<6>(dv, v);
      nz = 1;
    } else {
      double v[6];
      ld_n<6>(dv, v);
#pragma unroll
      for (int k = 0; k < 6; ++k) nz |= v[k] != 0.0;
    }
    if (nz && !w.nz) atomicOr(&w.nz, 1);
  }
}

// Span end: the best iterate back into vm, then (after the control kernel) the commit.
__global__ void k_w_restore(WaveArgs a) {
  const RoundItems R = round_items(a, kRangeBody, a.n_body);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.body[t];
    if (a.ctl[it.x].state != WS_END) continue;
    Ctx c = wave_ctx(a, it.x);
    double v[6];
    ld_n<6>(c.s.best + 6 * (size_t)it.y, v);
    st_n<6>(c.s.vm + 6 * (size_t)it.y, v);
  }
}

__global__ void k_w_commit(WaveArgs a) {
  const RoundItems R = round_items(a, kRangeDyn, a.n_dyn);
  for (int vi = gtid(); vi < R.n; vi += gthreads()) {
    const int t = R.at(vi);
    int2 it = a.dyn[t];
    const WaveCtl& w = a.ctl[it.x];
    if (!(w.flags & F_COMMIT)) continue;
    Ctx c = wave_ctx(a, it.x);
    op_commit(c, w.span, w.half, w.commit_converged != 0, it.y);
  }
}


// The elimination level by level (leaves to roots), then the back substitution (roots to leaves):
// levels of at most dev->tune_wave_narrow_level nodes take the warp kernels.
// NS: the kernels carry the Newton-Schulz pivot inverse (some island of the wave asks for it); without
// it they are the plain Gauss-Jordan kernels, whose register budgets the Newton-Schulz code would raise.
template <bool MIXED, bool NS>
void launch_solve_down(exg_device_s* dev, const WaveArgs& a, int first, int count, int r, cudaStream_t s) {
  constexpr int T = down_threads<MIXED && NS>();
  if (count <= dev->tune_wave_narrow_level)
    k_w_solve_down_warp<MIXED, NS><<<grid_for(dev, 32LL * count, 32 * kSolveWarps, 16), 32 * kSolveWarps, 0, s>>>(
        a, first, count, r);
  else
    k_w_solve_down<MIXED, NS><<<grid_for(dev, count, T, (256 / T) * dev->tune_wave_blocks_per_sm), T,
                                (MIXED && NS) ? 72 * T * sizeof(double) : 0, s>>>(a, first, count, r);
}

void launch_elimination(exg_device_s* dev, const WaveArgs& a, const std::vector<int>& level_ptr, bool mixed, bool ns,
                        cudaStream_t s) {
  const int nl = (int)level_ptr.size() - 1;
  const int narrow = dev->tune_wave_narrow_level;
  const int per = 2 * dev->tune_wave_blocks_per_sm;
  for (int L = nl - 1; L >= 0; --L) {
    const int first = level_ptr[L], count = level_ptr[L + 1] - first, r = kRangeLevel + L;
    if (mixed && ns) launch_solve_down<true, true>(dev, a, first, count, r, s);
    else if (mixed) launch_solve_down<true, false>(dev, a, first, count, r, s);
    else launch_solve_down<false, false>(dev, a, first, count, r, s);
  }
  for (int L = 1; L < nl; ++L) {
    const int first = level_ptr[L], count = level_ptr[L + 1] - first, r = kRangeLevel + L;
    if (count <= narrow)
      k_w_solve_up_warp<<<grid_for(dev, 32LL * count, 32 * kSolveWarps, 16), 32 * kSolveWarps, 0, s>>>(a, first,
                                                                                                     count, r);
    else
      k_w_solve_up<<<grid_for(dev, count, 128, per), 128, 0, s>>>(a, first, count, r);
  }
}

}  // namespace

// ── host: wave structure and rounds ──────────────────────────────────────────
bool NewtonWorld::wave_island(const IslandDesc& d) const {
  // block-LU islands (dynamic cycles) run on the island kernel
  return d.solver == 0 && d.m >= wave_min_dyn_ && d.n_levels <= wave_max_levels_;
}

int NewtonWorld::build_wave(cudaStream_t s) {
  std::vector<int> isl, dyn_first{0};
  std::vector<int2> body, dyn, joint, cell, cell_range;
  int max_levels = 0;
  for (int I = 0; I < (int)desc_.size(); ++I)
    if (alive_[I] && wave_island(desc_[I])) isl.push_back(I);
  for (int k = 0; k < (int)isl.size(); ++k) {
    const IslandDesc& d = desc_[isl[k]];
    for (int q = 0; q < d.nb; ++q) body.push_back(make_int2(k, q));
    for (int i = 0; i < d.m; ++i) dyn.push_back(make_int2(k, i));
    dyn_first.push_back((int)dyn.size());
    for (int q = 0; q < d.nj; ++q) joint.push_back(make_int2(k, q));
    // Cells in groups that read the same Jacobian slices: group p holds the diagonal of p and
    // (parent row, p col) — both read p's parent joints at p's end — and (child row, p col) of
    // every child c, which read c's joints at p's end, as the diagonal of p does. A slice's two
    // readers then run side by side (one pass from DRAM); cells are independent, so the order
    // changes no result.
    auto emit = [&](int t) {
      cell.push_back(make_int2(k, t));
      cell_range.push_back(make_int2(h_cell_ptr[d.cell_off + t], h_cell_ptr[d.cell_off + t + 1]));
    };
    std::vector<int> ch_first(d.m + 1, 0), ch_list(d.m);
    for (int i = 0; i < d.m; ++i)
      if (h_dn_parent[d.dyn_off + i] >= 0) ++ch_first[h_dn_parent[d.dyn_off + i] + 1];
    for (int i = 0; i < d.m; ++i) ch_first[i + 1] += ch_first[i];
    {
      std::vector<int> fill(ch_first.begin(), ch_first.end() - 1);
      for (int i = 0; i < d.m; ++i)
        if (h_dn_parent[d.dyn_off + i] >= 0) ch_list[fill[h_dn_parent[d.dyn_off + i]]++] = i;
    }
    for (int p = 0; p < d.m; ++p) {
      emit(3 * p);
      emit(3 * p + 2);
      if (h_dn_parent[d.dyn_off + p] < 0) emit(3 * p + 1);  // a root's: no terms
      for (int u = ch_first[p]; u < ch_first[p + 1]; ++u) emit(3 * ch_list[u] + 1);
    }
    max_levels = std::max(max_levels, d.n_levels);
  }
  // joint items grouped by law (a warp then evaluates one law), islands in order within a law
  auto law_of = [&](const int2& x) { return h_jl_law[desc_[isl[x.x]].joint_off + x.y]; };
  std::stable_sort(joint.begin(), joint.end(), [&](const int2& x, const int2& y) { return law_of(x) < law_of(y); });
  for (int L = 0; L <= 4; ++L)
    wave_law_first_[L] = (int)(std::lower_bound(joint.begin(), joint.end(), L,
                                                [&](const int2& x, int v) { return law_of(x) < v; }) - joint.begin());
  wave_law_first_[5] = (int)joint.size();  // items from first[4] on: the traced laws, dispatched at run time
  // nodes by elimination level across the wave's islands
  std::vector<std::vector<int2>> by(max_levels);
  for (int k = 0; k < (int)isl.size(); ++k) {
    const IslandDesc& d = desc_[isl[k]];
    for (int L = 0; L < d.n_levels; ++L)
      for (int u = h_lv_ptr[d.lv_off + L]; u < h_lv_ptr[d.lv_off + L + 1]; ++u)
        by[L].push_back(make_int2(k, h_lv_nodes[d.dyn_off + u]));
  }
  std::vector<int2> level;
  wave_level_ptr_.assign(1, 0);
  for (int L = 0; L < max_levels; ++L) {
    level.insert(level.end(), by[L].begin(), by[L].end());
    wave_level_ptr_.push_back((int)level.size());
  }
  // each range's per-slot item offsets (items of a range are in slot order)
  const int n_slots = (int)isl.size();
  wave_ranges_ = kRangeLevel + max_levels;
  std::vector<int> seg((size_t)wave_ranges_ * (n_slots + 1), 0);
  auto offsets = [&](int r, const std::vector<int2>& items, int first, int count) {
    int* o = seg.data() + (size_t)r * (n_slots + 1);
    for (int t = first; t < first + count; ++t) ++o[items[t].x + 1];
    for (int k = 0; k < n_slots; ++k) o[k + 1] += o[k];
  };
  offsets(kRangeBody, body, 0, (int)body.size());
  offsets(kRangeDyn, dyn, 0, (int)dyn.size());
  offsets(kRangeCell, cell, 0, (int)cell.size());
  for (int L = 0; L < 5; ++L) offsets(kRangeJoint + L, joint, wave_law_first_[L], wave_law_first_[L + 1] - wave_law_first_[L]);
  for (int L = 0; L < max_levels; ++L)
    offsets(kRangeLevel + L, level, wave_level_ptr_[L], wave_level_ptr_[L + 1] - wave_level_ptr_[L]);
  int rc = EXG_OK;
  auto up = [&](auto& d, const auto& h) {
    if (rc == EXG_OK) rc = d.assign(h.data(), (long long)h.size(), s);
  };
  std::vector<IslandDesc> wdesc;
  for (int I : isl) wdesc.push_back(desc_[I]);
  up(dw_isl_, isl);
  up(dw_desc_, wdesc);
  up(dw_dyn_first_, dyn_first);
  up(dw_body_, body);
  up(dw_dyn_, dyn);
  up(dw_joint_, joint);
  up(dw_cell_, cell);
  up(dw_cell_terms_, cell_range);
  up(dw_level_, level);
  up(dw_seg_, seg);
  if (rc == EXG_OK) rc = dw_act_.reserve(std::max(n_slots, 1), s);
  if (rc == EXG_OK) rc = dw_pre_.reserve(std::max<long long>((long long)seg.size(), 1), s);
  if (rc == EXG_OK) rc = dw_ctl_.reserve(std::max<long long>((long long)isl.size(), 1) * (long long)sizeof(WaveCtl), s);
  if (rc == EXG_OK) rc = dw_nodesq_.reserve(std::max<long long>((long long)dyn.size(), 1), s);
  if (rc == EXG_OK && dw_live_.cap == 0) {
    std::vector<int> z(kLiveCount, 0);
    rc = dw_live_.assign(z.data(), kLiveCount, s);
    seen_rounds_ = seen_dir_ = seen_end_ = 0;
  }
  if (rc != EXG_OK) return rc;
  n_wave_ = (int)isl.size();
  wave_counts_[0] = (int)body.size();
  wave_counts_[1] = (int)dyn.size();
  wave_counts_[2] = (int)joint.size();
  wave_counts_[3] = (int)cell.size();
  if (wave_graph_) cudaGraphExecDestroy(wave_graph_);
  wave_graph_ = nullptr;
  return EXG_OK;
}

int NewtonWorld::run_wave(exg_device_s* dev, DeviceWorld& w, cudaStream_t s) {
  if (n_wave_ == 0) return EXG_OK;
  WaveArgs a;
  a.A = arr;
  a.W = WorldRef{w.pose,    w.mom,    w.mass,   w.inertia, w.kinematic,  w.diagonal, w.pos_mass,
                 w.grav_partial, w.wparams, w.w_poff, w.w_splits, w.w_n, w.w_body_off, w.w_active, w.n};
  a.ctl = reinterpret_cast<WaveCtl*>(dw_ctl_.ptr);
  a.isl = dw_isl_.ptr;
  a.wdesc = dw_desc_.ptr;
  a.n_isl = n_wave_;
  a.body = dw_body_.ptr;
  a.n_body = wave_counts_[0];
  a.dyn = dw_dyn_.ptr;
  a.n_dyn = wave_counts_[1];
  a.joint = dw_joint_.ptr;
  a.n_joint = wave_counts_[2];
  a.cell = dw_cell_.ptr;
  a.cell_range = dw_cell_terms_.ptr;
  a.n_cell = wave_counts_[3];
  a.level = dw_level_.ptr;
  a.dyn_first = dw_dyn_first_.ptr;
  a.nodesq = dw_nodesq_.ptr;
  a.live = dw_live_.ptr;
  a.seg = dw_seg_.ptr;
  a.n_ranges = wave_ranges_;
  a.act = dw_act_.ptr;
  a.pre = dw_pre_.ptr;
  const int T = 256;
  const int g_isl = grid_for(dev, a.n_isl, T, 4);
  const int g_body = grid_for(dev, a.n_body, T, dev->tune_wave_blocks_per_sm);
  bool want_ns = false;  // some world asks for Newton-Schulz pivots (mixed path only)
  if (w.precision != EXG_PRECISION_F64)
    for (const exg_step_params_t& p : w.h_params) want_ns = want_ns || (p.newton_flags & EXG_NEWTON_NS_PIVOT) != 0;
  if (wave_graph_ && (wave_mixed_ != (w.precision != EXG_PRECISION_F64) || wave_ns_ != want_ns)) {
    cudaGraphExecDestroy(wave_graph_);
    wave_graph_ = nullptr;
  }
  wave_mixed_ = w.precision != EXG_PRECISION_F64;
  wave_ns_ = want_ns;
  int tok = prof_begin(dev, PROF_NEWTON_WAVE, s);
  k_w_init<<<g_isl, T, 0, s>>>(a);
  k_w_frame<<<std::min(a.n_isl, std::max(1, dev->sm_count) * 8), kFrameThreads, 0, s>>>(a);
  dev->launches.fetch_add(2, std::memory_order_relaxed);
  k_w_external<<<g_body, T, 0, s>>>(a);
  int rc = exg_after_launch(dev);
  if (rc != EXG_OK) return rc;
  static_assert(sizeof(WorldRef) <= sizeof(wave_graph_world_), "world snapshot too small");
  if (wave_graph_ && (std::memcmp(wave_graph_world_, &a.W, sizeof(WorldRef)) != 0 ||
                      wave_graph_tuning_ != dev->tune_wave_blocks_per_sm ||
                      wave_graph_narrow_ != dev->tune_wave_narrow_level || wave_graph_host_loop_ != wave_host_loop_)) {
    cudaGraphExecDestroy(wave_graph_);  // a world array moved since the capture
    wave_graph_ = nullptr;
  }
  if (!wave_graph_) {
    std::memcpy(wave_graph_world_, &a.W, sizeof(WorldRef));
    wave_graph_tuning_ = dev->tune_wave_blocks_per_sm;
    wave_graph_narrow_ = dev->tune_wave_narrow_level;
    wave_graph_host_loop_ = wave_host_loop_;
    rc = wave_host_loop_ ? build_wave_round_graph(dev, &a, s) : build_wave_graph(dev, &a, s);
    if (rc != EXG_OK) return rc;
  }
  if (!wave_host_loop_) {
    EXG_CUDA_TRY(cudaGraphLaunch(wave_graph_, s));
    prof_end(dev, tok, s);
    return EXG_OK;
  }
  // Host-driven form: one flat round graph (every section launched, islands that do not need it
  // skip it) replayed until a device counter says every island is done.
  int v[kLiveCount];
  int rounds = 0;
  for (;;) {
    const int batch = rounds < 4 ? 4 : 1;
    for (int r = 0; r < batch; ++r) {
      EXG_CUDA_TRY(cudaGraphLaunch(wave_graph_, s));
      dev->launches.fetch_add(wave_kernels_eval_ + wave_kernels_dir_ + wave_kernels_end_);
    }
    rounds += batch;
    EXG_CUDA_TRY(cudaMemcpyAsync(v, dw_live_.ptr, sizeof v, cudaMemcpyDeviceToHost, s));
    EXG_CUDA_TRY(cudaStreamSynchronize(s));
    if (v[kLiveIslands] == 0) break;
    if (rounds >= kMaxRoundsPerStep) return EXG_ERR_FATAL;
  }
  prof_end(dev, tok, s);
  last_wave_rounds_ = rounds;
  return EXG_OK;
}

// The host-driven form's round: the same kernels as the conditional graph's body, every section
// unconditional. For tools that do not follow kernels into conditional graph nodes (profilers).
int NewtonWorld::build_wave_round_graph(exg_device_s* dev, const void* args, cudaStream_t s) {
  const WaveArgs& a = *static_cast<const WaveArgs*>(args);
  const bool mixed = wave_mixed_;
  const int T = 256;
  const int g_isl = grid_for(dev, a.n_isl, T, 4);
  const int g_body = grid_for(dev, a.n_body, T, dev->tune_wave_blocks_per_sm);
  const int g_dyn = grid_for(dev, a.n_dyn, T, dev->tune_wave_blocks_per_sm);
  const int g_cell = grid_for(dev, 32LL * ((a.n_cell + 2) / 3), T, dev->tune_wave_blocks_per_sm);
  const int g_sum = std::min(a.n_isl, std::max(1, dev->sm_count) * 8);
  const int nl = (int)wave_level_ptr_.size() - 1;
  cudaGraph_t g;
  if (int rc = ensure_side()) return rc;
  EXG_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  k_w_round_items<<<1, kListThreads, 0, s>>>(a);
  k_w_begin<<<g_isl, T, 0, s>>>(a);
  k_w_start<<<g_body, T, 0, s>>>(a);
  k_w_pre<<<g_body, T, 0, s>>>(a);
  joints_forked(dev, &a, mixed, s);
  k_w_post<<<g_dyn, T, 0, s>>>(a);
  k_w_after_eval<<<g_isl, T, 0, s>>>(a);
  k_w_copy_bodies<<<g_body, T, 0, s>>>(a);
  if (mixed) k_w_assemble<true><<<g_cell, T, 0, s>>>(a);
  else k_w_assemble<false><<<g_cell, T, 0, s>>>(a);
  launch_elimination(dev, a, wave_level_ptr_, mixed, mixed && wave_ns_, s);
  k_w_nz<<<g_dyn, T, 0, s>>>(a);
  k_w_after_solve<<<g_isl, T, 0, s>>>(a);
  k_w_copy_bodies<<<g_body, T, 0, s>>>(a);
  k_w_restore<<<g_body, T, 0, s>>>(a);
  k_w_node_sq<<<g_dyn, T, 0, s>>>(a, 0);
  k_w_island_sum<<<g_sum, kSumThreads, 0, s>>>(a, 0);
  k_w_node_sq<<<g_dyn, T, 0, s>>>(a, 1);
  k_w_island_sum<<<g_sum, kSumThreads, 0, s>>>(a, 1);
  k_w_end<<<g_isl, T, 0, s>>>(a);
  k_w_commit<<<g_dyn, T, 0, s>>>(a);
  k_w_count_flat<<<1, 1024, 0, s>>>(a);
  cudaError_t le = cudaGetLastError();
  cudaError_t e = cudaStreamEndCapture(s, &g);
  EXG_CUDA_TRY(le);
  EXG_CUDA_TRY(e);
  cudaError_t ie = cudaGraphInstantiate(&wave_graph_, g, 0);
  cudaGraphDestroy(g);
  EXG_CUDA_TRY(ie);
  int joint_kernels = 0;
  for (int L = 0; L < 5; ++L)
    if (wave_law_first_[L + 1] > wave_law_first_[L]) joint_kernels += (L == LAW_TORSIONAL) ? 1 : 3;
  wave_kernels_eval_ = 7 + joint_kernels;  // round items, begin .. copy
  wave_kernels_dir_ = 1 + nl + (nl - 1) + 3;
  wave_kernels_end_ = 8;
  return EXG_OK;
}

int NewtonWorld::ensure_side() {
  if (!side_) EXG_CUDA_TRY(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  if (!fork_) EXG_CUDA_TRY(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  if (!join_) EXG_CUDA_TRY(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming));
  return EXG_OK;
}

// A round's joint tasks, captured: the Jacobian slices on s and, beside them on the side stream,
// the FP64 values; the side branch joins s again before anything that reads the values.
void NewtonWorld::joints_forked(exg_device_s* dev, const void* args, bool mixed, cudaStream_t s) {
  const WaveArgs& a = *static_cast<const WaveArgs*>(args);
  cudaEventRecord(fork_, s);
  cudaStreamWaitEvent(side_, fork_, 0);
  if (mixed) launch_joints_by_law<true>(dev, a, wave_law_first_, s, side_);
  else launch_joints_by_law<false>(dev, a, wave_law_first_, s, side_);
  cudaEventRecord(join_, side_);
  cudaStreamWaitEvent(s, join_, 0);
}

// The step's rounds as one graph: WHILE (some island unfinished) { evaluation; IF (some island
// needs a direction) { assembly, elimination, line-search start }; IF (some span ends) { commit } }.
// The conditions are set on the device (k_w_cond, k_w_count), so a step needs no host round trip.
int NewtonWorld::build_wave_graph(exg_device_s* dev, const void* args, cudaStream_t s) {
  const WaveArgs& a = *static_cast<const WaveArgs*>(args);
  const bool mixed = a.W.n >= 0 && wave_mixed_;
  const int T = 256;
  const int g_isl = grid_for(dev, a.n_isl, T, 4);
  const int g_body = grid_for(dev, a.n_body, T, dev->tune_wave_blocks_per_sm);
  const int g_dyn = grid_for(dev, a.n_dyn, T, dev->tune_wave_blocks_per_sm);
  const int g_cell = grid_for(dev, 32LL * ((a.n_cell + 2) / 3), T, dev->tune_wave_blocks_per_sm);
  const int g_sum = std::min(a.n_isl, std::max(1, dev->sm_count) * 8);
  const int nl = (int)wave_level_ptr_.size() - 1;
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  if (int rc = ensure_side()) return rc;
  cudaGraph_t G = nullptr;
  EXG_CUDA_TRY(cudaGraphCreate(&G, 0));
  struct Guard { cudaGraph_t g; ~Guard() { if (g) cudaGraphDestroy(g); } } guard{G};
  cudaGraphConditionalHandle h_loop, h_dir, h_end;
  EXG_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_loop, G, 1, cudaGraphCondAssignDefault));
  EXG_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_dir, G, 0, cudaGraphCondAssignDefault));
  EXG_CUDA_TRY(cudaGraphConditionalHandleCreate(&h_end, G, 0, cudaGraphCondAssignDefault));
  auto conditional = [&](cudaGraph_t parent, const cudaGraphNode_t* deps, size_t nd, cudaGraphConditionalHandle h,
                         cudaGraphConditionalNodeType type, cudaGraphNode_t* node, cudaGraph_t* body) {
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(node, parent, deps, nd, &p);
    if (e == cudaSuccess) *body = p.conditional.phGraph_out[0];
    return e;
  };
  // capture launches into `graph` after `deps`; returns the new tail
  std::vector<cudaGraphNode_t> tail;
  auto capture = [&](cudaGraph_t graph, const std::vector<cudaGraphNode_t>& deps, auto&& launches) -> cudaError_t {
    cudaError_t e = cudaStreamBeginCaptureToGraph(s, graph, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                                  mode);
    if (e != cudaSuccess) return e;
    launches();
    cudaError_t le = cudaGetLastError();
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t* d = nullptr;
    size_t n = 0;
    cudaError_t ie = cudaStreamGetCaptureInfo(s, &st, nullptr, nullptr, &d, &n);
    if (ie == cudaSuccess) tail.assign(d, d + n);
    cudaGraph_t out;
    cudaError_t ee = cudaStreamEndCapture(s, &out);
    return le != cudaSuccess ? le : (ie != cudaSuccess ? ie : ee);
  };
  cudaGraphNode_t loop, if_dir, if_end;
  cudaGraph_t B, BD, BE;
  EXG_CUDA_TRY(conditional(G, nullptr, 0, h_loop, cudaGraphCondTypeWhile, &loop, &B));
  // evaluation of every island at its iterate or probe
  EXG_CUDA_TRY(capture(B, {}, [&] {
    k_w_round_items<<<1, kListThreads, 0, s>>>(a);
    k_w_begin<<<g_isl, T, 0, s>>>(a);
    k_w_start<<<g_body, T, 0, s>>>(a);
    k_w_pre<<<g_body, T, 0, s>>>(a);
    joints_forked(dev, &a, mixed, s);
    k_w_post<<<g_dyn, T, 0, s>>>(a);
    k_w_after_eval<<<g_isl, T, 0, s>>>(a);
    k_w_copy_bodies<<<g_body, T, 0, s>>>(a);
    k_w_cond<<<1, 1024, 0, s>>>(a, h_dir, WS_DIR, kLiveTotalDir);
  }));
  EXG_CUDA_TRY(conditional(B, tail.data(), tail.size(), h_dir, cudaGraphCondTypeIf, &if_dir, &BD));
  // direction: assembly, elimination level by level, back substitution, line-search start
  EXG_CUDA_TRY(capture(BD, {}, [&] {
    if (mixed) k_w_assemble<true><<<g_cell, T, 0, s>>>(a);
    else k_w_assemble<false><<<g_cell, T, 0, s>>>(a);
    launch_elimination(dev, a, wave_level_ptr_, mixed, mixed && wave_ns_, s);
    k_w_nz<<<g_dyn, T, 0, s>>>(a);
    k_w_after_solve<<<g_isl, T, 0, s>>>(a);
    k_w_copy_bodies<<<g_body, T, 0, s>>>(a);
  }));
  EXG_CUDA_TRY(capture(B, {if_dir}, [&] { k_w_cond<<<1, 1024, 0, s>>>(a, h_end, WS_END, kLiveTotalEnd); }));
  EXG_CUDA_TRY(conditional(B, tail.data(), tail.size(), h_end, cudaGraphCondTypeIf, &if_end, &BE));
  // span end: the best iterate back, the stiffness signal, sub-division or commit
  EXG_CUDA_TRY(capture(BE, {}, [&] {
    k_w_restore<<<g_body, T, 0, s>>>(a);
    k_w_node_sq<<<g_dyn, T, 0, s>>>(a, 0);
    k_w_island_sum<<<g_sum, kSumThreads, 0, s>>>(a, 0);
    k_w_node_sq<<<g_dyn, T, 0, s>>>(a, 1);
    k_w_island_sum<<<g_sum, kSumThreads, 0, s>>>(a, 1);
    k_w_end<<<g_isl, T, 0, s>>>(a);
    k_w_commit<<<g_dyn, T, 0, s>>>(a);
  }));
  EXG_CUDA_TRY(capture(B, {if_end}, [&] { k_w_count<<<1, 1024, 0, s>>>(a, h_loop); }));
  EXG_CUDA_TRY(cudaGraphInstantiate(&wave_graph_, G, 0));
  int joint_kernels = 0;
  for (int L = 0; L < 5; ++L)
    if (wave_law_first_[L + 1] > wave_law_first_[L]) joint_kernels += (L == LAW_TORSIONAL) ? 1 : 3;
  wave_kernels_eval_ = 7 + joint_kernels + 2;  // round items, begin .. copy, cond(dir), cond(end), count
  wave_kernels_dir_ = 1 + nl + (nl - 1) + 3;
  wave_kernels_end_ = 7;
  return EXG_OK;
}

// After a synchronised step: the wave's launched-kernel count and whether a step hit the round
// cap (reported as EXG_ERR_FATAL).
int NewtonWorld::wave_after_steps(exg_device_s* dev) {
  if (n_wave_ == 0 || dw_live_.cap < kLiveCount || wave_graph_host_loop_) return EXG_OK;
  int v[kLiveCount];
  EXG_CUDA_TRY(cudaMemcpy(v, dw_live_.ptr, sizeof v, cudaMemcpyDeviceToHost));
  last_wave_rounds_ = v[kLiveRounds];
  const long long dr = v[kLiveTotalRounds] - seen_rounds_, dd = v[kLiveTotalDir] - seen_dir_,
                  de = v[kLiveTotalEnd] - seen_end_;
  seen_rounds_ = v[kLiveTotalRounds];
  seen_dir_ = v[kLiveTotalDir];
  seen_end_ = v[kLiveTotalEnd];
  dev->launches.fetch_add((uint64_t)(dr * wave_kernels_eval_ + dd * wave_kernels_dir_ + de * wave_kernels_end_));
  return v[kLiveOverflow] ? EXG_ERR_FATAL : EXG_OK;
}
