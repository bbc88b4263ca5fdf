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

struct IslandDesc {
  int world;             // the world (of the batch) the island belongs to
  int body_off, nb;      // island bodies: isl_body[body_off .. body_off+nb)
  int joint_off, nj;     // island joints: isl_joint[joint_off .. joint_off+nj)
  int dyn_off, m;        // dynamic nodes: dn_*[dyn_off .. dyn_off+m)
  int lv_off, n_levels;  // level pointers lv_ptr[lv_off .. lv_off+n_levels+1)
  int cell_off;          // cell_ptr[cell_off .. cell_off + 3m + 1)
  int inc_off;           // ib_inc_ptr[inc_off .. inc_off + nb + 1)
  long long scratch_off; // doubles
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
  double* scratch;
  int* stats;              // per island: spans, newton iterations, max depth, fatal
  double* residual;        // per island: last span's best residual
  long long* phase_cycles; // [kPhases] SM clock cycles per phase, summed over islands and steps
};
// Phases of the device Newton step, for the cycle counters.
enum NewtonPhase { PH_PRE = 0, PH_JACOBIAN = 1, PH_POST = 2, PH_ASSEMBLE = 3, PH_SOLVE = 4, PH_LINE_SEARCH = 5,
                   PH_COMMIT = 6, PH_OTHER = 7, kPhases = 8 };

class NewtonWorld {
 public:
  int init(exg_device_s* dev, DeviceWorld& w, const exg_body_t* bodies, const exg_joint_t* joints, const exg_step_params_t& p);
  // Enqueue one step of every island (no host synchronisation; graph-capturable).
  int enqueue(exg_device_s* dev, DeviceWorld& w, cudaStream_t s);
  // Aggregate the last step's per-island counters, over all islands (world < 0) or one world.
  int read_stats(int world, exg_world_stats_t* stats);
  int n_islands_total() const { return n_islands; }
  // Summed SM cycles per phase since the world was created (kPhases values).
  int read_phase_cycles(long long* out);
  ~NewtonWorld();

 private:
  int n_islands = 0;
  int max_nb = 0;
  std::vector<void*> allocs;
  NewtonDeviceArrays arr{};
  std::vector<int> island_order;  // islands sorted by size, largest first
  std::vector<int> island_world;
  int* d_queue = nullptr;         // island work queue (largest first) and its head counter
  int* d_head = nullptr;
};

double host_world_energy(const exg_body_t* b, int n, const exg_joint_t* joints, int nj, const exg_step_params_t& p);
