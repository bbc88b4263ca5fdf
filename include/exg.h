/*
 * exg.h — C ABI of the B200 per-step dynamics path (all-pairs gravity, joint force laws,
 * implicit mid-point Newton step).
 *
 * This is the drop-in boundary a host binds instead of the reference's Vulkan device layer
 * and GPU-resident world storage. Every entry point takes plain pointers and sizes and
 * returns an `int` status (EXG_OK = 0, negative = error; `exg_status_string` names it).
 * Host arrays are ordinary CPU memory; entry points whose parameter is named `d_*` take
 * device pointers on the device the handle was created on.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   - rembrandt::GpuAccelerator (crates/rembrandt/src/lib.rs:77-243)      -> exg_device_*
 *   - aristotle::World storage + WorldKey slots (crates/aristotle/src/world.rs:400-650)
 *                                                                        -> exg_world_* (device buffers)
 *   - newton::Accelerator stage calls (crates/newton/src/accelerator/mod.rs:649-964)
 *                                                                        -> exg_eval_joints, exg_gravity_forces
 *   - Mechanism::step / Driver::step (crates/newton/src/mechanism/mechanism.rs:526,
 *     crates/newton/src/driver.rs:76)                                    -> exg_world_step, exg_batch_step
 *   - joint-law registration by shader name (crates/newton/src/accelerator/mod.rs:118-132,
 *     crates/joints/src/lib.rs:246-253)                                  -> exg_law_lookup
 *   - EvalError / StructureError (crates/newton/src/error.rs:11-28,
 *     crates/newton/src/mechanism/mechanism.rs:21-58)                    -> exg_status codes
 */
#ifndef EXG_H
#define EXG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EXG_ABI_VERSION 2

#if defined(__GNUC__)
#define EXG_API __attribute__((visibility("default")))
#else
#define EXG_API
#endif

/* ── status codes ─────────────────────────────────────────────────────────── */
typedef enum {
  EXG_OK = 0,
  /* EvalError (crates/newton/src/error.rs:11-28) */
  EXG_ERR_NO_SHADER = -1,       /* NoShader: unknown joint-law name or id */
  EXG_ERR_TRAP = -2,            /* Trap: a kernel refused its input. Not returned here: records a
                                 * kernel would refuse are checked before any kernel runs and
                                 * refused with EXG_ERR_INVALID_ARGUMENT */
  EXG_ERR_FATAL = -3,           /* Fatal: a guarded site fired (non-finite state) */
  EXG_ERR_WORKER_GONE = -4,     /* WorkerGone: the request loop has shut down */
  EXG_ERR_BACKEND = -5,         /* Backend: a CUDA call failed */
  /* StructureError (crates/newton/src/mechanism/mechanism.rs:21-58), kept so that a host's mapping
   * of the reference's errors stays total. This library returns none of the four: calls on one
   * handle exclude each other, so a structural change (exg_batch_set_joints, a kinematic flip in
   * exg_world_set_bodies, exg_pool_admit/release) waits for a step in flight on the handle instead
   * of being refused mid-epoch; body records are copied into a handle, so no body belongs to two;
   * a handle is bound to its device when created; and no call registers a world twice. */
  EXG_ERR_EPOCH_IN_PROGRESS = -10,
  EXG_ERR_ALREADY_OWNED = -11,
  EXG_ERR_FOREIGN_ACCELERATOR = -12,
  EXG_ERR_DUPLICATE_MECHANISM = -13,
  /* storage misuse, which panics in the reference (crates/aristotle/src/world.rs:246-264) */
  EXG_ERR_INVALID_ARGUMENT = -20,
  EXG_ERR_OUT_OF_MEMORY = -21,
  EXG_ERR_UNSUPPORTED = -22,
  EXG_ERR_TIMEOUT = -23,
  EXG_ERR_NO_DEVICE = -24
} exg_status;

/* ── records (host layout == device layout) ───────────────────────────────── */

/* One rigid body (crates/newton/src/body.rs:32-63). `pose` is the motor in the reference's
 * slot order (even blades by increasing bitmask: 1, e12, e13, e23, e1e0, e2e0, e3e0, e123e0 in
 * bit terms 0,3,5,6,9,10,12,15; crates/clifford/src/pga3/motor.rs:119-147). `momentum` is the
 * BODY-frame momentum (force xyz, torque xyz). `inertia` is the 3x3 angular tensor, row-major
 * (crates/newton/src/inertia.rs:145-156); `diagonal` = 1 reads only its diagonal. `size` is the
 * gravity core radius, (mass/4)^(1/3) by default (body.rs:70-77). A kinematic body has a
 * prescribed velocity equal to its momentum read as a twist (inertia.rs:160-170). */
typedef struct {
  double pose[8];
  double momentum[6];
  double mass;
  double inertia[9];
  double size;
  int32_t kinematic;
  int32_t diagonal;
} exg_body_t;

/* One joint edge (crates/joints/src/lib.rs:47-60): law id, the two body indices and the law's
 * parameters in its canonical flatten order (crates/joints/src/lib.rs:273-298). */
typedef struct {
  int32_t law;
  int32_t a;
  int32_t b;
  int32_t reserved;
  double params[10];
} exg_joint_t;

typedef enum {
  EXG_LAW_SIMPLE_SPRING_DAMPER = 0,        /* "SimpleSpringDamper", 10 params */
  EXG_LAW_CRITICALLY_DAMPED_WARPED = 1,    /* "CriticallyDampedWarped", 10 params */
  EXG_LAW_PERPENDICULAR_DAMPER_WARPED = 2, /* "PerpendicularDamperWarped", 2 params */
  EXG_LAW_TORSIONAL_DAMPER_WARPED = 3      /* "TorsionalDamperWarped", 1 param */
} exg_law;

typedef enum { EXG_EXPLICIT_EULER = 0, EXG_SYMPLECTIC_EULER = 1, EXG_LIE_EULER = 2, EXG_NEWTON = 3 } exg_integrator;
typedef enum { EXG_GRAVITY_OFF = 0, EXG_GRAVITY_SIZE_CORE = 1, EXG_GRAVITY_PLUMMER = 2 } exg_gravity_law;
/* F64: every stage in double precision (the plain path). MIXED: gravity pair terms and the Newton
 * Jacobian's derivative slices in FP32; poses, momenta, joint wrench values, the residual and
 * convergence test, the assembled system and its solve in FP64. Gravity takes pair separations
 * from double-single (hi + lo FP32) positions, so a close pair's separation is accurate to its
 * own FP32 rounding. MIXED_FAST: as MIXED with single FP32 positions relative to the gravity tile's
 * reference body (faster; the rounding of that reference distance then enters close pairs, which
 * dense clusters amplify over many steps). */
typedef enum { EXG_PRECISION_F64 = 0, EXG_PRECISION_MIXED = 1, EXG_PRECISION_MIXED_FAST = 2 } exg_precision;

/* Step configuration: Epoch dt/warp (crates/aristotle/src/epoch.rs:17-60), the integrator
 * (crates/newton/src/integrator/implicit/mod.rs:44-49), the gravity field and the Newton
 * tolerance (relative per-block residual; the reference hard-codes 1e-4,
 * crates/newton/src/integrator/implicit/newton.rs:799-805). */
/* newton_flags bit 0: assemble the Newton matrix with the exact derivative of the mid-point
 * retraction on the pose columns (-half^2/2) instead of the reference's -half^2
 * (crates/newton/src/integrator/implicit/cache.rs:509-520). Either matrix leads to the same
 * converged step; the exact one converges in fewer iterations. */
#define EXG_NEWTON_EXACT_POSE_FACTOR 1
/* newton_flags bit 1 (mixed precisions only): invert the elimination's 6x6 pivot blocks by
 * Newton-Schulz (the reference's iteration, crates/newton/src/integrator/implicit/newton.rs:209-327,
 * at block size): warm-started from the node's inverse of the previous solve in the step, FP32
 * steps where the block moved, one FP64 correction (exg_pivot_inverse states the details); without
 * it the pivots take FP64 Gauss-Jordan. Both converge to the same step. */
#define EXG_NEWTON_NS_PIVOT 2

typedef struct {
  int32_t integrator;
  int32_t gravity_law;
  int32_t precision;
  int32_t newton_flags;
  double G;
  double softening; /* Plummer epsilon */
  double dt;
  double warp;
  double tol;
  int32_t max_newton; /* per span; the reference uses 32 (newton.rs:355) */
  int32_t reserved1;
  /* UniformField (crates/newton/src/field.rs:17-47): a constant world acceleration; every body
   * gets the world force m * field_accel (kinematic bodies, mass 0, none), added to the external
   * wrench beside gravity. Zero: no field. */
  double field_accel[3];
} exg_step_params_t;

/* Per-world counters of the last step. */
typedef struct {
  int64_t steps;
  int32_t last_spans;            /* dt sub-spans taken (newton.rs:543-683) */
  int32_t last_newton_iterations;
  int32_t max_depth_reached;
  int32_t fatal;                 /* non-zero after a non-finite residual was committed */
  double last_residual;          /* worst relative residual^2 of the last span */
} exg_world_stats_t;

typedef struct exg_device_s* exg_device_t;
typedef struct exg_world_s* exg_world_t;

/* ── device (replaces rembrandt::GpuAccelerator::new, crates/rembrandt/src/lib.rs:98-158) ── */
EXG_API int exg_device_create(int32_t ordinal, exg_device_t* out);
/* Refused (EXG_ERR_INVALID_ARGUMENT) while world handles made on the device are alive: destroy
 * them (and servers) first. */
EXG_API int exg_device_destroy(exg_device_t dev);
EXG_API int exg_device_synchronize(exg_device_t dev);
/* Number of kernels this library launched on the device so far. */
EXG_API int exg_device_kernel_launches(exg_device_t dev, uint64_t* out);
EXG_API const char* exg_status_string(int status);
/* The CUDA stream (cudaStream_t) every call on this device is ordered on. */
EXG_API int exg_device_stream(exg_device_t dev, void** out);
/* In-library profiler: when enabled, each kernel launch is bracketed by CUDA events on the device
 * stream (worlds then launch directly instead of through a CUDA graph). Kinds: 0 gravity,
 * 1 joints, 2 explicit integrate, 3 Newton step (island kernel), 4 body pre, 5 Newton step (wave
 * schedule). Enabling or disabling resets the
 * totals; read returns the summed device time and the launch count of one kind. */
EXG_API int exg_device_profile(exg_device_t dev, int32_t enable);
EXG_API int exg_device_profile_read(exg_device_t dev, int32_t kind, double* total_ms, int64_t* launches);
EXG_API int exg_abi_version(void);

/* Launch-shape tuning of a device (exgame_b200.autotune measures and sets these). No result
 * depends on them: they change how work is spread over the SMs, not the arithmetic.
 *   GRAVITY_CTAS_PER_SM  persistent CTAs per SM of the mixed gravity kernel (1..64, default 32)
 *   WAVE_BLOCKS_PER_SM   grid cap per SM of the wave schedule's data kernels (1..32, default 16)
 *   WAVE_MIN_BODIES      wave threshold given to world handles created afterwards (default 32;
 *                        the island kernel and the wave give identical results) */
#define EXG_TUNE_GRAVITY_CTAS_PER_SM 1
#define EXG_TUNE_WAVE_BLOCKS_PER_SM 2
#define EXG_TUNE_WAVE_MIN_BODIES 3
/*   WAVE_NARROW_LEVEL   elimination levels of the wave with at most this many nodes take one warp per
 *                       node, wider ones one thread per node (1..2^30, default 8192; the two
 *                       kernels give the same bits) */
#define EXG_TUNE_WAVE_NARROW_LEVEL 4
EXG_API int exg_device_set_tuning(exg_device_t dev, int32_t key, int32_t value);
EXG_API int exg_device_get_tuning(exg_device_t dev, int32_t key, int32_t* value);

/* ── law registry (MessageKind::from((shader_name, jacobian)), accelerator/mod.rs:118-132) ── */
EXG_API int exg_law_lookup(const char* shader_name, int32_t* law_out, int32_t* n_params_out);

/* ── world: device-resident bodies and joints (aristotle::World + Mechanism) ── */
EXG_API int exg_world_create(exg_device_t dev, const exg_body_t* bodies, int32_t n_bodies, const exg_joint_t* joints,
                     int32_t n_joints, const exg_step_params_t* params, exg_world_t* out);
EXG_API int exg_world_destroy(exg_world_t w);
/* Advance n_steps steps (Mechanism::step per step; crates/newton/src/mechanism/mechanism.rs:526-602). */
EXG_API int exg_world_step(exg_world_t w, int32_t n_steps);
EXG_API int exg_world_get_bodies(exg_world_t w, exg_body_t* out, int32_t n_bodies);
EXG_API int exg_world_set_bodies(exg_world_t w, const exg_body_t* bodies, int32_t n_bodies);
/* The dynamic state alone, in the record order of exg_world_get/set_bodies: per body pose[8] then
 * momentum[6] (14 doubles, 112 B; the first two fields of exg_body_t). Mass, inertia, size and
 * flags stay as they are on the device, so a loop that feeds states in and reads them back each
 * step (Mechanism::step with the host reading poses, crates/newton/src/mechanism/mechanism.rs:526)
 * moves 112 B per body each way instead of a record's 208 B. */
EXG_API int exg_world_get_state(exg_world_t w, double* state, int32_t n_bodies);
EXG_API int exg_world_set_state(exg_world_t w, const double* state, int32_t n_bodies);
EXG_API int exg_world_stats(exg_world_t w, exg_world_stats_t* out);

/* ── batch: many independent worlds of uneven size stepped together (Driver::step over many
 * mechanisms, crates/newton/src/driver.rs:76-80; Accelerator::epoch, accelerator/mod.rs:613-630).
 * World k owns body_counts[k] consecutive records of `bodies` and joint_counts[k] consecutive
 * records of `joints`, whose body indices are local to world k. Every world has its own step
 * parameters; all must share one precision. The returned handle is an exg_world_t: exg_world_step
 * advances every world by one step per call step, and exg_world_get/set_bodies see the whole
 * batch (world k at offset sum(body_counts[0..k))). A world of one is exg_world_create. */
EXG_API int exg_batch_create(exg_device_t dev, int32_t n_worlds, const int32_t* body_counts, const int32_t* joint_counts,
                             const exg_body_t* bodies, const exg_joint_t* joints, const exg_step_params_t* params,
                             exg_world_t* out);
EXG_API int exg_batch_get_world(exg_world_t w, int32_t world, exg_body_t* out, int32_t n_bodies);
EXG_API int exg_batch_set_world(exg_world_t w, int32_t world, const exg_body_t* bodies, int32_t n_bodies);
EXG_API int exg_batch_world_stats(exg_world_t w, int32_t world, exg_world_stats_t* out);
/* New joints for one world of a batch or pool (world 0 of a single world): joint records with
 * world-local body indices, replacing the world's joint list. Adding a joint between two islands
 * merges them, removing one may split an island (Islands::connect / detach,
 * crates/newton/src/mechanism/islands.rs:166-299; Mechanism::split / merge,
 * crates/newton/src/mechanism/mechanism.rs:326-434); the islands and the solver's structure are
 * rebuilt before the next step (cache.rs:689-788). The bodies keep their state on the device.
 * An island whose dynamic bodies form a cycle takes the block-LU solve. All or nothing:
 * EXG_ERR_OUT_OF_MEMORY (no room in the handle's joint capacity: a world or batch handle holds the
 * joint count it was created with, a pool max_joints) or a bad record leaves the world as it was. */
EXG_API int exg_batch_set_joints(exg_world_t w, int32_t world, const exg_joint_t* joints, int32_t n_joints);
/* The epoch of one world (world 0 of a single world) for the following steps: its dt and warp
 * (Epoch::standalone(dt, warp), crates/aristotle/src/epoch.rs:17-60; the reference passes the
 * epoch to every Mechanism::step, so a host with a variable frame time sets it before each step).
 * dt > 0 and finite, warp >= 1; no structural change, nothing is rebuilt. */
EXG_API int exg_batch_set_epoch(exg_world_t w, int32_t world, double dt, double warp);
/* ── pool: worlds admitted into and released from fixed-capacity device arrays ──
 * The serving form of a batch: state stays resident while worlds come and go. A released slot's
 * ranges are reused by later admissions; exg_world_step advances every admitted world. The
 * batch accessors (exg_batch_get/set_world, exg_batch_world_stats) take the slot returned by
 * exg_pool_admit. Admission fails with EXG_ERR_OUT_OF_MEMORY when no free range or slot fits. */
typedef struct {
  int64_t max_bodies;
  int64_t max_joints;
  int32_t max_worlds;
  int32_t precision; /* every admitted world must use this precision */
} exg_pool_config_t;
typedef struct {
  int32_t worlds_used;
  int32_t worlds_capacity;
  int64_t largest_free_bodies;
  int64_t largest_free_joints;
} exg_pool_usage_t;
EXG_API int exg_pool_create(exg_device_t dev, const exg_pool_config_t* cfg, exg_world_t* out);
EXG_API int exg_pool_admit(exg_world_t pool, const exg_body_t* bodies, int32_t n_bodies, const exg_joint_t* joints,
                           int32_t n_joints, const exg_step_params_t* params, int32_t* slot_out);
EXG_API int exg_pool_release(exg_world_t pool, int32_t slot);
EXG_API int exg_pool_free(exg_world_t pool, exg_pool_usage_t* out);
/* Step budget of one admitted world: it takes `steps` more steps of the pool and then holds its
 * state while the others go on (-1, the default at admission: no limit). */
EXG_API int exg_pool_set_steps(exg_world_t pool, int32_t slot, int32_t steps);
/* Steps left per slot for slots [0, n_slots) (-1: no limit; 0 for a free slot or a world whose
 * budget is spent). */
EXG_API int exg_pool_steps_left(exg_world_t pool, int32_t* out, int32_t n_slots);
/* Page-locked host memory for record buffers: exg_world_get/set_bodies and the batch accessors copy
 * from and into such buffers at the link's full rate (pageable buffers are staged by the driver). */
EXG_API int exg_host_alloc(size_t bytes, void** out);
EXG_API int exg_host_free(void* ptr);

/* Device bytes a world holds while admitted to a pool: its body and joint rows, gravity partial
 * sums and, for the implicit integrator, its island structure and per-step scratch (an upper
 * estimate: every body counted as dynamic, one island). */
EXG_API int exg_world_footprint(int32_t n_bodies, int32_t n_joints, const exg_step_params_t* params, int64_t* bytes);

/* ── serving: a continuous-batching request loop over a pool ──
 * Replaces the reference's single GPU-owner worker thread (crates/newton/src/accelerator/mod.rs:
 * 1010-1155) for whole simulation requests: any thread submits a world and a step count; one
 * worker thread admits requests in arrival order while the admitted worlds' footprints stay
 * within hbm_budget_bytes and the pool has room, steps the pool in ticks of at most
 * steps_per_tick steps, and publishes each world when its steps are done. Each world takes exactly
 * its requested steps with the arithmetic it has alone. EXG_ERR_WORKER_GONE after the loop stopped
 * on a device error (EvalError::WorkerGone, crates/newton/src/error.rs:11-28). */
#define EXG_PENDING 1 /* poll: the request is queued or running */
typedef struct exg_server_s* exg_server_t;
typedef struct {
  int64_t hbm_budget_bytes; /* bound on the sum of admitted worlds' exg_world_footprint */
  int64_t max_bodies;       /* pool capacities */
  int64_t max_joints;
  int32_t max_worlds;
  int32_t precision;        /* every request must use this precision */
  int32_t steps_per_tick;   /* steps between admissions / completions */
  /* 1 (or 0): one pool. 2: the capacities split between two pools on streams of their own, each
   * stepped by its own worker thread, so one pool's admissions, uploads and read-backs overlap the
   * other pool's tick on the GPU. */
  int32_t pools;
} exg_server_config_t;
typedef struct {
  int64_t steps;
  int32_t n_bodies;
  int32_t status;    /* EXG_PENDING, EXG_OK or the failure */
  double queued_s;   /* submit to admission */
  double latency_s;  /* submit to completion (to now while pending) */
} exg_request_info_t;
typedef struct {
  int64_t submitted, completed, failed, ticks, steps_launched, body_steps;
  int32_t queued, running, peak_running, reserved;
  int64_t resident_bytes, peak_resident_bytes;
  double busy_s, elapsed_s, p50_latency_s, p99_latency_s, mean_latency_s;
} exg_server_stats_t;
EXG_API int exg_server_create(exg_device_t dev, const exg_server_config_t* cfg, exg_server_t* out);
EXG_API int exg_server_submit(exg_server_t server, const exg_body_t* bodies, int32_t n_bodies, const exg_joint_t* joints,
                              int32_t n_joints, const exg_step_params_t* params, int32_t steps, uint64_t* id);
/* EXG_PENDING while queued or running; otherwise the request's status, its final bodies copied to
 * out (when out is not NULL; n must equal its body count) and the request forgotten. */
EXG_API int exg_server_poll(exg_server_t server, uint64_t id, exg_body_t* out, int32_t n, exg_request_info_t* info);
/* poll after waiting up to timeout_ms for the request to finish (EXG_ERR_TIMEOUT otherwise) */
EXG_API int exg_server_wait(exg_server_t server, uint64_t id, int32_t timeout_ms, exg_body_t* out, int32_t n,
                            exg_request_info_t* info);
EXG_API int exg_server_stats(exg_server_t server, exg_server_stats_t* out);
EXG_API int exg_server_reset_stats(exg_server_t server);
EXG_API int exg_server_destroy(exg_server_t server);
/* ── schedule options of a world handle ──
 * Implicit islands run one of two device schedules with the same per-item arithmetic: the island
 * kernel (one CTA per island, the whole step in one launch) or the wave schedule (every phase a
 * grid-wide kernel over all large islands, rounds of a captured graph). An island takes the wave
 * schedule when it has at least EXG_OPT_WAVE_MIN_BODIES dynamic bodies and at most
 * EXG_OPT_WAVE_MAX_LEVELS elimination levels. The choice depends on the island alone, so a world
 * steps the same in every batch with the same options. */
#define EXG_OPT_WAVE_MIN_BODIES 1
#define EXG_OPT_WAVE_MAX_LEVELS 2
#define EXG_OPT_LAST_WAVE_ROUNDS 3 /* read only: rounds the wave schedule ran in the last step */
/* 1: the wave's rounds are replayed from the host (one flat graph per round, a device counter read
 * between them) instead of running inside one conditional graph; identical results. For profilers
 * that do not follow kernels into conditional graph nodes. */
#define EXG_OPT_WAVE_HOST_ROUNDS 4
/* 1: the handle runs on a stream of its own, and calls on it no longer wait for calls on other
 * handles, so host threads holding different handles overlap their copies and steps on the GPU
 * (the accelerator's worker serialises all flushes, crates/newton/src/accelerator/mod.rs:1044;
 * here only a handle is single-writer). 0 (default): the device's stream, shared with every other
 * handle on it; calls on such handles take turns. */
#define EXG_OPT_OWN_STREAM 5
/* Read only, after a step: the most and the fewest nodes on one elimination level of the wave
 * schedule, across the handle's wave islands (the wave eliminates levels wider than 8192 nodes one
 * thread per node, narrower ones one warp per node); 0 without wave islands. */
#define EXG_OPT_WAVE_LEVEL_MAX_WIDTH 6
#define EXG_OPT_WAVE_LEVEL_MIN_WIDTH 7
EXG_API int exg_world_set_option(exg_world_t world, int32_t option, int64_t value);
EXG_API int exg_world_get_option(exg_world_t world, int32_t option, int64_t* value);
/* The CUDA stream (cudaStream_t) the handle's work runs on, for events around its calls. */
EXG_API int exg_world_stream(exg_world_t world, void** stream_out);
/* SM clock cycles the implicit step spent per phase since the handle was created, summed over
 * islands: [0] PRE, [1] joint values + Jacobian, [2] gather + POST, [3] assembly, [4] linear
 * solve, [5] line search, [6] commit, [7] other. Zero for worlds without implicit islands. */
EXG_API int exg_world_phase_cycles(exg_world_t w, int64_t out[8]);
/* ── solver structure read-back ──
 * The islands of one implicit world (world 0 of a single-world handle, a batch index or a pool
 * slot) and, per island, the integer maps the kernels index by, copied back from the device. These
 * are the reference's per-island topology and gather maps (crates/newton/src/mechanism/islands.rs;
 * bake_incidence, crates/newton/src/accelerator/mod.rs:289-331; the solver cache's dynamic order,
 * crates/newton/src/integrator/implicit/cache.rs:566-573, 885-897), for checking them integer for
 * integer. Islands come in order of their first body; an explicit world has none.
 *   ISLAND_BODIES  per island body: its world-local body index (ascending)
 *   JOINT_ENDS     per island joint, three ints: law, end a, end b (island-local body indices)
 *   ORDER          per island body: its index among the island's dynamic bodies, -1 if kinematic
 *   INCIDENCE_PTR  per island body plus one: offsets into INCIDENCE
 *   INCIDENCE      per gathered term, in gather order: island joint * 2 + end (0 = a, 1 = b)
 *   PARENT         per dynamic body: its parent in the elimination order's tree, -1 for a root
 *   ISLAND_JOINTS  per island joint: its world-local joint index (ascending)
 * `cap` is the capacity of out in ints; *len receives the length even when it exceeds cap
 * (EXG_ERR_INVALID_ARGUMENT then). */
#define EXG_STRUCT_ISLAND_BODIES 1
#define EXG_STRUCT_JOINT_ENDS 2
#define EXG_STRUCT_ORDER 3
#define EXG_STRUCT_INCIDENCE_PTR 4
#define EXG_STRUCT_INCIDENCE 5
#define EXG_STRUCT_PARENT 6
#define EXG_STRUCT_ISLAND_JOINTS 7
EXG_API int exg_world_island_count(exg_world_t w, int32_t world, int32_t* n_islands);
EXG_API int exg_world_island_structure(exg_world_t w, int32_t world, int32_t island, int32_t kind, int32_t* out,
                                       int32_t cap, int32_t* len);

/* Total energy: kinetic + gravity + joint potential (crates/newton/tests/energy_drift_repro.rs:123-149). */
EXG_API int exg_world_energy(exg_world_t w, double* out);

/* ── typed slot storage (aristotle::World per-type storage, crates/aristotle/src/world.rs) ──
 * One storage holds elements of elem_bytes (a multiple of 4, at most 65536) in one device buffer
 * of `capacity` slots (WorldBuilder::with_storage / capacity, world.rs:498-538). A key is the slot
 * index and the slot's generation (MapKey; WorldKey::raw_index, world.rs:479-487). Inserting takes
 * the lowest free slot (the reference keeps its free list in slot order, RawMap::insert / remove,
 * world.rs:300-370); a fresh slot starts at generation 0 and freeing bumps the slot's generation, so
 * a stale or freed key is refused (EXG_ERR_INVALID_ARGUMENT) by read, write and free. Inserting into
 * a full buffer grows it geometrically: every live slot is copied to the same position and the
 * storage's generation is bumped (RawMap::grow, world.rs:189-211; World::generation, world.rs:
 * 625-633), so indices survive growth while a holder of the old buffer pointer learns that it must
 * re-bind. Device memory is not host-mapped: read and write are explicit copies; the _n forms move
 * many slots in one gather or scatter kernel. A storage counts as a handle of its device. */
typedef struct exg_storage_s* exg_storage_t;
typedef struct {
  uint32_t index;
  uint32_t generation;
} exg_slot_key_t;
typedef struct {
  void* buffer;        /* the device buffer (valid while the generation below is current) */
  int64_t elem_bytes;
  int64_t capacity;    /* slots the buffer holds */
  int64_t len;         /* slots ever handed out (live or free) */
  int64_t live;        /* live keys */
  uint64_t generation; /* bumped by every growth */
} exg_storage_info_t;
EXG_API int exg_storage_create(exg_device_t dev, int64_t elem_bytes, int64_t capacity, exg_storage_t* out);
EXG_API int exg_storage_destroy(exg_storage_t st);
EXG_API int exg_slot_alloc(exg_storage_t st, const void* value, exg_slot_key_t* key);
EXG_API int exg_slot_free(exg_storage_t st, exg_slot_key_t key);
EXG_API int exg_slot_read(exg_storage_t st, exg_slot_key_t key, void* out);
EXG_API int exg_slot_write(exg_storage_t st, exg_slot_key_t key, const void* value);
EXG_API int exg_slot_read_n(exg_storage_t st, const exg_slot_key_t* keys, int32_t n, void* out);
/* The batch's writes run unordered on the device, so a batch naming one slot twice is refused
 * before anything is written (the one-writer ledger below). All keys are checked first: a stale
 * key refuses the batch too. */
EXG_API int exg_slot_write_n(exg_storage_t st, const exg_slot_key_t* keys, int32_t n, const void* values);
EXG_API int exg_storage_info(exg_storage_t st, exg_storage_info_t* out);

/* ── one-writer ledger (crates/newton/src/accelerator/shaders.rs:321-390) ──
 * The check every batch of unordered writes passes before it runs: each of slots[0, n) must lie in
 * [0, n_slots) and no slot may be named twice. EXG_OK, or EXG_ERR_BACKEND (the reference refuses
 * the flush with EvalError::Backend) with exg_status_string naming the slot and *first_clash the
 * position of the first offending entry. The library runs it on its own scatter maps whenever a
 * world's structure is rebuilt (island bodies, gathered joint ends, assembly terms, factor blocks),
 * and on every batched slot write. Host only: no device needed. */
EXG_API int exg_ledger_check(const int32_t* slots, int64_t n, int64_t n_slots, int64_t* first_clash);

/* ── host-side motor utilities (no device needed; the same algebra the kernels use) ── */
/* Twist::exp(dt) of (linear xyz, angular xyz) -> motor (crates/clifford/src/pga3/screw.rs:297-301). */
EXG_API int exg_motor_exp(const double twist[6], double dt, double out[8]);
/* "first a, then b" (Motor::compose, crates/clifford/src/pga3/motor.rs:157-159). */
EXG_API int exg_motor_compose(const double a[8], const double b[8], double out[8]);
EXG_API int exg_motor_inverse(const double a[8], double out[8]);
/* World coordinates of the local point p under motor m (joints/src/lib.rs:258-263). */
EXG_API int exg_motor_apply_point(const double m[8], const double p[3], double out[3]);
/* Screw transport under m: covariant = 0 for a twist (Ad), 1 for a wrench (coAd)
 * (crates/clifford/src/pga3/screw.rs:94-105). */
EXG_API int exg_screw_transport(const double s[6], const double m[8], int32_t covariant, double out[6]);
/* Array forms for building large worlds: out[k] = exp(twists[k] * dt) and out[k] = compose(a[k], b[k]). */
EXG_API int exg_motor_exp_n(int64_t count, const double* twists, double dt, double* out);
EXG_API int exg_motor_compose_n(int64_t count, const double* a, const double* b, double* out);

/* ── stage API on device pointers (the Accelerator's stage calls) ─────────── */
/* Joint kernels K1-K8 (crates/newton/build.rs:874-973): for each joint k, inputs are the two
 * poses (8 doubles each, d_pose[8*body]), the two WORLD twists (6 doubles each, d_vel[6*body]);
 * output is d_out[12*k] = [force a, torque a, force b, torque b] when jacobian == 0, or the
 * 300-double block d_out[300*k] = 12 components x [value, d/d(axis 0..23)] (axes: pose A,
 * pose B, vel A, vel B; each lin xyz then ang xyz) when jacobian != 0. */
EXG_API int exg_eval_joints(exg_device_t dev, const exg_joint_t* d_joints, int32_t n_joints, const double* d_pose,
                    const double* d_vel, double dt, double warp, int32_t jacobian, double* d_out);
/* The implicit solve's 6x6 pivot inverse on n row-major blocks d_blocks[36*k] -> d_out[36*k]
 * (the block inverse of the reference's Newton-Schulz solve, crates/newton/src/integrator/implicit/
 * newton.rs:209-327: seed_transpose, refine_inverse, the warm start). precision MIXED or
 * MIXED_FAST: the inverse the mixed path takes with EXG_NEWTON_NS_PIVOT. With warm != 0, d_out
 * holds on entry an earlier inverse of each block (the block before a small change): where its
 * FP64 residual max|I - D X| is at most 1e-4, one FP64 Newton-Schulz correction; otherwise FP32
 * Newton-Schulz steps held in registers on the diagonally scaled block (seeded with the earlier
 * inverse where its residual is below 1/2, else with the identity or the reference's transposed
 * seed) and one FP64 correction, FP64 Gauss-Jordan for a block whose FP32 residual stays above
 * 1e-3. F64: FP64 Gauss-Jordan with partial pivoting (the plain path's). form 0 runs one thread
 * per block (a wide elimination level's form), 1 one warp per block (a narrow level's and the
 * island kernel's); both give the same bits. d_steps (may be NULL) receives per block the FP32
 * steps taken (0 where the warm correction sufficed), -1 where the block fell back to Gauss-Jordan,
 * 0 on F64. EXG_ERR_FATAL if a block is singular (its output is then not finite). */
EXG_API int exg_pivot_inverse(exg_device_t dev, const double* d_blocks, int32_t n, int32_t precision, int32_t form,
                              int32_t warm, double* d_out, int32_t* d_steps);
/* All-pairs gravity (crates/newton/src/gravity.rs:110-140, 438-450): d_pos_mass holds
 * [x, y, z, m] per body, d_size the core radius (SIZE_CORE law), output d_force[3*i] is the
 * world force on body i. precision MIXED runs the FP32 kernel on double-single separations,
 * MIXED_FAST the single-FP32 one, F64 the double kernel; any other precision code is
 * EXG_ERR_INVALID_ARGUMENT. */
EXG_API int exg_gravity_forces(exg_device_t dev, const double* d_pos_mass, const double* d_size, int32_t n, int32_t law,
                       double G, double softening, int32_t precision, double* d_force);

/* ── gravity without allocation ────────────────────────────────────────────────
 * Same result as exg_gravity_forces, for callers that must not allocate device memory: code that
 * runs under a strict memory budget or a pre-sized pool, or code whose allocator may not be called
 * at that point (for example a host that reserves all device memory up front). This entry point
 * has no counterpart in the reference.
 * Its working memory (work items, per-split partial sums and the scheduler counter) is a fixed
 * array compiled into the library: every GPU that loads the library holds about 3.2 MB of it until
 * the process exits. Bodies are limited to EXG_NOALLOC_MAX_BODIES; larger n returns
 * EXG_ERR_INVALID_ARGUMENT before any work is queued.
 * The first call on a device looks up that array's device address (once per device, with the
 * device current); make that first call before capturing any stream into a CUDA graph. The address
 * belongs to the device's primary context: exg_device_create forgets it, so after a
 * cudaDeviceReset create a new device handle before the next call.
 * Every call on a device uses the same array and leaves its contents behind; the call resets what
 * must start at zero. Two calls whose GPU work overlaps (from different threads or streams) race
 * on the array. The call returns after its work has finished. */
#define EXG_NOALLOC_MAX_BODIES 16384
EXG_API int exg_gravity_forces_noalloc(exg_device_t dev, const double* d_pos_mass, const double* d_size, int32_t n,
                                       int32_t law, double G, double softening, int32_t precision, double* d_force);

#ifdef __cplusplus
}
#endif
#endif /* EXG_H */
