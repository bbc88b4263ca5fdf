// Implicit mid-point Newton step on the device (crates/newton/src/integrator/implicit/newton.rs:334-861).
//
// Host side: NewtonWorld partitions a world into islands (connected components of the joint
// graph, crates/newton/src/mechanism/islands.rs), builds each island's solve structure once
// (dynamic-body order, incidence in the reference's gather order, the elimination tree rooted
// at the tree centre, assembly cell lists) and owns the device scratch. Device side: one CTA
// per island runs the whole step — spans, Newton iterations, line search, sub-division and the
// motor update — without returning to the host.
#pragma once
#include "exg_internal.cuh"
#include "slab.cuh"

struct IslandDesc {
  int world;             // the world (of the batch) the island belongs to
  int body_off, nb;      // island bodies: isl_body[body_off .. body_off+nb)
  int joint_off, nj;     // island joints: isl_joint[joint_off .. joint_off+nj)
  int dyn_off, m;        // dynamic nodes: dn_*[dyn_off .. dyn_off+m)
  int lv_off, n_levels;  // level pointers lv_ptr[lv_off .. lv_off+n_levels+1)
  int cell_off;          // cell_ptr[cell_off .. cell_off + 3m + 1)
  int inc_off;           // ib_inc_ptr[inc_off .. inc_off + nb + 1)
  long long scratch_off; // doubles
  // Linear solve: 0 = block elimination on the island's tree (its dynamic bodies form a forest),
  // 1 = block LU on a minimum-degree elimination order with fill (dynamic cycles). For solver 1
  // the island's blocks are D[0..m) then, per off-diagonal slot s (a pair k < j in elimination
  // order, fill included), Up = A(k, j) and Lo = A(j, k) at blocks m + 2s and m + 2s + 1; levels
  // (lv_*) run from the first eliminated nodes up, and the gn_* arrays hold the factorization's
  // update lists.
  int solver;
  int n_slots;           // off-diagonal slots (solver 1)
  int gen_off;           // gn_rop_ptr / gn_slot_ptr [gen_off .. gen_off + m + 1)
  int gen_lv_off;        // gn_lgrp [gen_lv_off .. gen_lv_off + n_levels + 1)
  int gen_slot_off;      // gn_slot_col [gen_slot_off .. gen_slot_off + n_slots)
};

struct NewtonDeviceArrays {
  const IslandDesc* desc;
  const int* isl_body;     // global body index per island body
  const int* jl_law;       // per island joint: law
  const int* jl_a;         // per island joint: island-local a
  const int* jl_b;         // per island joint: island-local b
  const double* jl_params; // per island joint: 10 params
  const int* ib_order;     // per island body: dynamic node index or -1
  const int* ib_inc_ptr;   // per island body incidence CSR (relative to the island's joint list)
  const int* ib_inc_ref;   // local joint * 2 + end
  const int* dn_body;      // per dynamic node: island-local body
  const int* dn_parent;    // per dynamic node: parent node or -1
  const int* lv_ptr;       // nodes grouped by elimination level
  const int* lv_nodes;
  const int* ch_ptr;       // children CSR per node (island-relative node ids)
  const int* ch_idx;
  const int* cell_ptr;     // assembly terms per (node, kind)
  const int* cell_terms;   // local joint * 4 + row_end * 2 + col_end
  // solver 1 (block LU): per level, its update groups (absolute offsets into gn_grp); a group is
  // (target block, first op, end op) over gn_ops, each op (left block, right block): target -=
  // left * right, in order; per node, its right-hand-side updates (absolute into gn_rops, each (the
  // scaled block S = A(k, p) D_p^-1, p)) and its slots (island-relative, columns in gn_slot_col).
  const int* gn_lgrp;
  const int4* gn_grp;
  const int2* gn_ops;
  const int* gn_rop_ptr;
  const int2* gn_rops;
  const int* gn_slot_ptr;
  const int* gn_slot_col;
  double* scratch;
  int* stats;              // per island: spans, newton iterations, max depth, fatal
  double* residual;        // per island: last span's best residual
  long long* phase_cycles; // [kPhases] SM clock cycles per phase, summed over islands and steps
};
// Phases of the device Newton step, for the cycle counters.
enum NewtonPhase { PH_PRE = 0, PH_JACOBIAN = 1, PH_POST = 2, PH_ASSEMBLE = 3, PH_SOLVE = 4, PH_LINE_SEARCH = 5,
                   PH_COMMIT = 6, PH_OTHER = 7, kPhases = 8 };

// Islands of the implicit worlds of a pool. Worlds are added and removed one at a time; their
// island structure is appended to device arrays that only grow, and each island's per-step
// scratch is a range of one scratch array (contents do not persist across steps, so the array is
// reallocated without copying when it must grow).
class NewtonWorld {
 public:
  ~NewtonWorld();
  // Build the islands of one world (bodies and joints local to the world; its bodies live at
  // body_off in the pool) and queue them for stepping.
  int add_world(exg_device_s* dev, int slot, int body_off, const exg_body_t* bodies, int n, const exg_joint_t* joints,
                int nj);
  void remove_world(int slot);
  // Whether the world's kinematic flags differ from `bodies` (its islands were built from them).
  bool kin_differs(int slot, const exg_body_t* bodies, int n) const;
  // The kinematic flags the world's islands were built from.
  std::vector<char> kin_of(int slot) const;
  // Rebuild the world's islands for new kinematic flags (same joints); on a structure error the
  // world keeps its previous islands.
  int rebuild_world(int slot, const std::vector<char>& kin);
  // Rebuild the world's islands for a new joint list (world-local body indices; same bodies);
  // on a structure error the world keeps its previous islands.
  int replace_joints(int slot, const exg_joint_t* joints, int nj);
  // Upload pending structure and the island queue (host synchronous; call outside stream capture).
  int sync(exg_device_s* dev, cudaStream_t s);
  bool dirty() const { return dirty_; }
  // Enqueue one step of every live island (no host synchronisation; graph-capturable once synced).
  int enqueue(exg_device_s* dev, DeviceWorld& w, cudaStream_t s);
  // Aggregate the last step's per-island counters, over all islands (world < 0) or one world.
  int read_stats(int world, exg_world_stats_t* stats);
  // Summed SM cycles per phase since creation (kPhases values).
  int read_phase_cycles(long long* out);
  int live_islands() const { return n_live_; }
  // Islands of one world (a slot of the pool), in island order (ascending first body).
  int island_count(int slot) const;
  // One array of island k's solver structure, copied back from the device arrays the kernels
  // read (the kinds of exg_world_island_structure); *len its length. Host synchronous; the
  // structure must be synced.
  int read_structure(int slot, int k, int kind, int* out, int cap, int* len);
  // Islands with at least min_dyn dynamic bodies and at most max_levels elimination levels take
  // the wave schedule (newton_wave.cu); the others the island kernel.
  void set_wave_threshold(int min_dyn, int max_levels) {
    wave_min_dyn_ = min_dyn;
    wave_max_levels_ = max_levels;
    dirty_ = true;
  }
  int wave_min_dyn() const { return wave_min_dyn_; }
  int wave_max_levels() const { return wave_max_levels_; }
  bool has_wave() const { return n_wave_ > 0; }
  // The wave schedule's step (host synchronous between rounds; call outside stream capture,
  // after the step's other kernels on the same stream).
  int run_wave(exg_device_s* dev, DeviceWorld& w, cudaStream_t s);
  // After the stream is synchronised: launched-kernel accounting, round-cap check.
  int wave_after_steps(exg_device_s* dev);
  int last_wave_rounds() const { return last_wave_rounds_; }
  // Widest (or narrowest) elimination level of the wave, in nodes; 0 without wave islands.
  int wave_level_width(bool widest) const {
    int best = 0;
    for (size_t L = 0; L + 1 < wave_level_ptr_.size(); ++L) {
      int wd = wave_level_ptr_[L + 1] - wave_level_ptr_[L];
      if (L == 0 || (widest ? wd > best : wd < best)) best = wd;
    }
    return best;
  }
  // Rounds driven from the host (one flat round graph per launch) instead of the conditional graph:
  // the same arithmetic, for profilers that do not follow kernels into conditional graph nodes.
  void set_wave_host_loop(bool on) { wave_host_loop_ = on; }
  bool wave_host_loop() const { return wave_host_loop_; }

 private:
  struct WorldSrc {  // what rebuilding a world's islands needs
    bool live = false;
    int body_off = 0;
    std::vector<char> kin;
    std::vector<exg_joint_t> joints;
  };
  int build_world(int slot, const WorldSrc& src);
  int rebuild_from(int slot, WorldSrc next);  // all or nothing
  void compact();
  bool wave_island(const IslandDesc& d) const;
  int build_wave(cudaStream_t s);
  // wave schedule
  int wave_min_dyn_ = 32, wave_max_levels_ = 64;
  int n_cta_ = 0, n_wave_ = 0;
  int wave_counts_[4] = {0, 0, 0, 0};  // body, dynamic node, joint and cell items
  int wave_law_first_[6] = {0, 0, 0, 0, 0, 0};  // joint items of law L: [first[L], first[L+1]); L = 4: traced laws
  std::vector<int> wave_level_ptr_;
  DevArr<int> dw_isl_, dw_dyn_first_, dw_live_;
  // per item range (body, dynamic node, cell, joint law 0..4, elimination level 0..): each slot's
  // first item in it (n_wave_ + 1 offsets); the round's listed slots and their item prefixes
  DevArr<int> dw_seg_, dw_act_, dw_pre_;
  int wave_ranges_ = 0;
  DevArr<IslandDesc> dw_desc_;  // island descriptors in wave-slot order
  DevArr<int2> dw_body_, dw_dyn_, dw_joint_, dw_cell_, dw_level_;
  DevArr<int2> dw_cell_terms_;  // per cell item: its term range in cell_terms (absolute)
  DevArr<unsigned char> dw_ctl_;
  DevArr<double> dw_nodesq_;
  cudaGraphExec_t wave_graph_ = nullptr;
  unsigned char wave_graph_world_[160] = {0};  // the world arrays the round graph was captured with
  int build_wave_graph(exg_device_s* dev, const void* args, cudaStream_t s);
  int build_wave_round_graph(exg_device_s* dev, const void* args, cudaStream_t s);
  // the side stream and events of the forked joint tasks (made before any capture)
  int ensure_side();
  void joints_forked(exg_device_s* dev, const void* args, bool mixed, cudaStream_t s);
  cudaStream_t side_ = nullptr;
  cudaEvent_t fork_ = nullptr, join_ = nullptr;
  bool wave_host_loop_ = false, wave_graph_host_loop_ = false;
  bool wave_mixed_ = false;
  bool wave_ns_ = false;  // the wave's elimination kernels carry the Newton-Schulz pivot inverse
  int wave_kernels_eval_ = 0, wave_kernels_dir_ = 0, wave_kernels_end_ = 0;
  long long seen_rounds_ = 0, seen_dir_ = 0, seen_end_ = 0;
  int wave_graph_tuning_ = 0;  // the launch-shape tuning the round graph was captured with
  int wave_graph_narrow_ = 0;
  int last_wave_rounds_ = 0;
  std::vector<WorldSrc> src_;
  bool dirty_ = true;
  int n_live_ = 0;
  // host structure (append-only)
  std::vector<IslandDesc> desc_;
  std::vector<char> alive_;
  std::vector<long long> scratch_len_;
  std::vector<int> h_isl_body, h_jl_law, h_jl_a, h_jl_b, h_ib_order, h_ib_inc_ptr, h_ib_inc_ref, h_dn_body, h_dn_parent,
      h_lv_ptr, h_lv_nodes, h_ch_ptr, h_ch_idx, h_cell_ptr, h_cell_terms;
  std::vector<double> h_jl_params;
  std::vector<int> h_jl_id;  // per island joint: the world-local joint index (host only)
  std::vector<int> h_gn_lgrp, h_gn_rop_ptr, h_gn_slot_ptr, h_gn_slot_col;
  std::vector<int4> h_gn_grp;
  std::vector<int2> h_gn_ops, h_gn_rops;
  std::vector<std::vector<int>> world_islands_;
  // device mirrors
  DevArr<IslandDesc> d_desc;
  DevArr<int> d_isl_body, d_jl_law, d_jl_a, d_jl_b, d_ib_order, d_ib_inc_ptr, d_ib_inc_ref, d_dn_body, d_dn_parent,
      d_lv_ptr, d_lv_nodes, d_ch_ptr, d_ch_idx, d_cell_ptr, d_cell_terms;
  DevArr<int> d_gn_lgrp, d_gn_rop_ptr, d_gn_slot_ptr, d_gn_slot_col;
  DevArr<int4> d_gn_grp;
  DevArr<int2> d_gn_ops, d_gn_rops;
  DevArr<double> d_jl_params, d_scratch, d_residual;
  DevArr<int> d_stats, d_queue;
  DevArr<long long> d_phase;
  RangeAllocator scratch_alloc_;
  NewtonDeviceArrays arr{};
};

// Upper estimate of the device bytes an implicit world's islands hold (one island, all dynamic).
long long newton_footprint_bytes(int nb, int nj);

double host_world_energy(const exg_body_t* b, int n, const exg_joint_t* joints, int nj, const exg_step_params_t& p);
