// Generated by include/rust/gen_ffi.py from include/exg.h; do not edit by hand.
//! Raw bindings of the B200 per-step dynamics library (libexg.so, include/exg.h).
//! Every entry point returns an exg_status (EXG_OK = 0, negative = error); see the header
//! for each call's contract.
#![allow(non_camel_case_types, non_upper_case_globals, non_snake_case, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

pub const EXG_ABI_VERSION: c_int = 2;
pub const EXG_NEWTON_EXACT_POSE_FACTOR: c_int = 1;
pub const EXG_NEWTON_NS_PIVOT: c_int = 2;
pub const EXG_TUNE_GRAVITY_CTAS_PER_SM: c_int = 1;
pub const EXG_TUNE_WAVE_BLOCKS_PER_SM: c_int = 2;
pub const EXG_TUNE_WAVE_MIN_BODIES: c_int = 3;
pub const EXG_TUNE_WAVE_NARROW_LEVEL: c_int = 4;
pub const EXG_PENDING: c_int = 1;
pub const EXG_OPT_WAVE_MIN_BODIES: c_int = 1;
pub const EXG_OPT_WAVE_MAX_LEVELS: c_int = 2;
pub const EXG_OPT_LAST_WAVE_ROUNDS: c_int = 3;
pub const EXG_OPT_WAVE_HOST_ROUNDS: c_int = 4;
pub const EXG_OPT_OWN_STREAM: c_int = 5;
pub const EXG_OPT_WAVE_LEVEL_MAX_WIDTH: c_int = 6;
pub const EXG_OPT_WAVE_LEVEL_MIN_WIDTH: c_int = 7;
pub const EXG_STRUCT_ISLAND_BODIES: c_int = 1;
pub const EXG_STRUCT_JOINT_ENDS: c_int = 2;
pub const EXG_STRUCT_ORDER: c_int = 3;
pub const EXG_STRUCT_INCIDENCE_PTR: c_int = 4;
pub const EXG_STRUCT_INCIDENCE: c_int = 5;
pub const EXG_STRUCT_PARENT: c_int = 6;
pub const EXG_STRUCT_ISLAND_JOINTS: c_int = 7;
pub const EXG_NOALLOC_MAX_BODIES: c_int = 16384;
pub const EXG_OK: c_int = 0;
pub const EXG_ERR_NO_SHADER: c_int = -1;
pub const EXG_ERR_TRAP: c_int = -2;
pub const EXG_ERR_FATAL: c_int = -3;
pub const EXG_ERR_WORKER_GONE: c_int = -4;
pub const EXG_ERR_BACKEND: c_int = -5;
pub const EXG_ERR_EPOCH_IN_PROGRESS: c_int = -10;
pub const EXG_ERR_ALREADY_OWNED: c_int = -11;
pub const EXG_ERR_FOREIGN_ACCELERATOR: c_int = -12;
pub const EXG_ERR_DUPLICATE_MECHANISM: c_int = -13;
pub const EXG_ERR_INVALID_ARGUMENT: c_int = -20;
pub const EXG_ERR_OUT_OF_MEMORY: c_int = -21;
pub const EXG_ERR_UNSUPPORTED: c_int = -22;
pub const EXG_ERR_TIMEOUT: c_int = -23;
pub const EXG_ERR_NO_DEVICE: c_int = -24;
pub const EXG_LAW_SIMPLE_SPRING_DAMPER: c_int = 0;
pub const EXG_LAW_CRITICALLY_DAMPED_WARPED: c_int = 1;
pub const EXG_LAW_PERPENDICULAR_DAMPER_WARPED: c_int = 2;
pub const EXG_LAW_TORSIONAL_DAMPER_WARPED: c_int = 3;
pub const EXG_EXPLICIT_EULER: c_int = 0;
pub const EXG_SYMPLECTIC_EULER: c_int = 1;
pub const EXG_LIE_EULER: c_int = 2;
pub const EXG_NEWTON: c_int = 3;
pub const EXG_GRAVITY_OFF: c_int = 0;
pub const EXG_GRAVITY_SIZE_CORE: c_int = 1;
pub const EXG_GRAVITY_PLUMMER: c_int = 2;
pub const EXG_PRECISION_F64: c_int = 0;
pub const EXG_PRECISION_MIXED: c_int = 1;
pub const EXG_PRECISION_MIXED_FAST: c_int = 2;

#[repr(C)]
pub struct exg_device_s {
    _private: [u8; 0],
}
pub type exg_device_t = *mut exg_device_s;
#[repr(C)]
pub struct exg_world_s {
    _private: [u8; 0],
}
pub type exg_world_t = *mut exg_world_s;
#[repr(C)]
pub struct exg_server_s {
    _private: [u8; 0],
}
pub type exg_server_t = *mut exg_server_s;
#[repr(C)]
pub struct exg_storage_s {
    _private: [u8; 0],
}
pub type exg_storage_t = *mut exg_storage_s;

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_body_t {
    pub pose: [f64; 8],
    pub momentum: [f64; 6],
    pub mass: f64,
    pub inertia: [f64; 9],
    pub size: f64,
    pub kinematic: i32,
    pub diagonal: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_joint_t {
    pub law: i32,
    pub a: i32,
    pub b: i32,
    pub reserved: i32,
    pub params: [f64; 10],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_step_params_t {
    pub integrator: i32,
    pub gravity_law: i32,
    pub precision: i32,
    pub newton_flags: i32,
    pub G: f64,
    pub softening: f64,
    pub dt: f64,
    pub warp: f64,
    pub tol: f64,
    pub max_newton: i32,
    pub reserved1: i32,
    pub field_accel: [f64; 3],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_world_stats_t {
    pub steps: i64,
    pub last_spans: i32,
    pub last_newton_iterations: i32,
    pub max_depth_reached: i32,
    pub fatal: i32,
    pub last_residual: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_pool_config_t {
    pub max_bodies: i64,
    pub max_joints: i64,
    pub max_worlds: i32,
    pub precision: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_pool_usage_t {
    pub worlds_used: i32,
    pub worlds_capacity: i32,
    pub largest_free_bodies: i64,
    pub largest_free_joints: i64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_server_config_t {
    pub hbm_budget_bytes: i64,
    pub max_bodies: i64,
    pub max_joints: i64,
    pub max_worlds: i32,
    pub precision: i32,
    pub steps_per_tick: i32,
    pub pools: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_request_info_t {
    pub steps: i64,
    pub n_bodies: i32,
    pub status: i32,
    pub queued_s: f64,
    pub latency_s: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_server_stats_t {
    pub submitted: i64,
    pub completed: i64,
    pub failed: i64,
    pub ticks: i64,
    pub steps_launched: i64,
    pub body_steps: i64,
    pub queued: i32,
    pub running: i32,
    pub peak_running: i32,
    pub reserved: i32,
    pub resident_bytes: i64,
    pub peak_resident_bytes: i64,
    pub busy_s: f64,
    pub elapsed_s: f64,
    pub p50_latency_s: f64,
    pub p99_latency_s: f64,
    pub mean_latency_s: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_slot_key_t {
    pub index: u32,
    pub generation: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct exg_storage_info_t {
    pub buffer: *mut c_void,
    pub elem_bytes: i64,
    pub capacity: i64,
    pub len: i64,
    pub live: i64,
    pub generation: u64,
}

#[link(name = "exg")]
extern "C" {
    pub fn exg_device_create(ordinal: i32, out: *mut exg_device_t) -> c_int;
    pub fn exg_device_destroy(dev: exg_device_t) -> c_int;
    pub fn exg_device_synchronize(dev: exg_device_t) -> c_int;
    pub fn exg_device_kernel_launches(dev: exg_device_t, out: *mut u64) -> c_int;
    pub fn exg_status_string(status: c_int) -> *const c_char;
    pub fn exg_device_stream(dev: exg_device_t, out: *mut *mut c_void) -> c_int;
    pub fn exg_device_profile(dev: exg_device_t, enable: i32) -> c_int;
    pub fn exg_device_profile_read(dev: exg_device_t, kind: i32, total_ms: *mut f64, launches: *mut i64) -> c_int;
    pub fn exg_abi_version() -> c_int;
    pub fn exg_device_set_tuning(dev: exg_device_t, key: i32, value: i32) -> c_int;
    pub fn exg_device_get_tuning(dev: exg_device_t, key: i32, value: *mut i32) -> c_int;
    pub fn exg_law_lookup(shader_name: *const c_char, law_out: *mut i32, n_params_out: *mut i32) -> c_int;
    pub fn exg_world_create(dev: exg_device_t, bodies: *const exg_body_t, n_bodies: i32, joints: *const exg_joint_t, n_joints: i32, params: *const exg_step_params_t, out: *mut exg_world_t) -> c_int;
    pub fn exg_world_destroy(w: exg_world_t) -> c_int;
    pub fn exg_world_step(w: exg_world_t, n_steps: i32) -> c_int;
    pub fn exg_world_get_bodies(w: exg_world_t, out: *mut exg_body_t, n_bodies: i32) -> c_int;
    pub fn exg_world_set_bodies(w: exg_world_t, bodies: *const exg_body_t, n_bodies: i32) -> c_int;
    pub fn exg_world_get_state(w: exg_world_t, state: *mut f64, n_bodies: i32) -> c_int;
    pub fn exg_world_set_state(w: exg_world_t, state: *const f64, n_bodies: i32) -> c_int;
    pub fn exg_world_stats(w: exg_world_t, out: *mut exg_world_stats_t) -> c_int;
    pub fn exg_batch_create(dev: exg_device_t, n_worlds: i32, body_counts: *const i32, joint_counts: *const i32, bodies: *const exg_body_t, joints: *const exg_joint_t, params: *const exg_step_params_t, out: *mut exg_world_t) -> c_int;
    pub fn exg_batch_get_world(w: exg_world_t, world: i32, out: *mut exg_body_t, n_bodies: i32) -> c_int;
    pub fn exg_batch_set_world(w: exg_world_t, world: i32, bodies: *const exg_body_t, n_bodies: i32) -> c_int;
    pub fn exg_batch_world_stats(w: exg_world_t, world: i32, out: *mut exg_world_stats_t) -> c_int;
    pub fn exg_batch_set_joints(w: exg_world_t, world: i32, joints: *const exg_joint_t, n_joints: i32) -> c_int;
    pub fn exg_batch_set_epoch(w: exg_world_t, world: i32, dt: f64, warp: f64) -> c_int;
    pub fn exg_pool_create(dev: exg_device_t, cfg: *const exg_pool_config_t, out: *mut exg_world_t) -> c_int;
    pub fn exg_pool_admit(pool: exg_world_t, bodies: *const exg_body_t, n_bodies: i32, joints: *const exg_joint_t, n_joints: i32, params: *const exg_step_params_t, slot_out: *mut i32) -> c_int;
    pub fn exg_pool_release(pool: exg_world_t, slot: i32) -> c_int;
    pub fn exg_pool_free(pool: exg_world_t, out: *mut exg_pool_usage_t) -> c_int;
    pub fn exg_pool_set_steps(pool: exg_world_t, slot: i32, steps: i32) -> c_int;
    pub fn exg_pool_steps_left(pool: exg_world_t, out: *mut i32, n_slots: i32) -> c_int;
    pub fn exg_host_alloc(bytes: usize, out: *mut *mut c_void) -> c_int;
    pub fn exg_host_free(ptr: *mut c_void) -> c_int;
    pub fn exg_world_footprint(n_bodies: i32, n_joints: i32, params: *const exg_step_params_t, bytes: *mut i64) -> c_int;
    pub fn exg_server_create(dev: exg_device_t, cfg: *const exg_server_config_t, out: *mut exg_server_t) -> c_int;
    pub fn exg_server_submit(server: exg_server_t, bodies: *const exg_body_t, n_bodies: i32, joints: *const exg_joint_t, n_joints: i32, params: *const exg_step_params_t, steps: i32, id: *mut u64) -> c_int;
    pub fn exg_server_poll(server: exg_server_t, id: u64, out: *mut exg_body_t, n: i32, info: *mut exg_request_info_t) -> c_int;
    pub fn exg_server_wait(server: exg_server_t, id: u64, timeout_ms: i32, out: *mut exg_body_t, n: i32, info: *mut exg_request_info_t) -> c_int;
    pub fn exg_server_stats(server: exg_server_t, out: *mut exg_server_stats_t) -> c_int;
    pub fn exg_server_reset_stats(server: exg_server_t) -> c_int;
    pub fn exg_server_destroy(server: exg_server_t) -> c_int;
    pub fn exg_world_set_option(world: exg_world_t, option: i32, value: i64) -> c_int;
    pub fn exg_world_get_option(world: exg_world_t, option: i32, value: *mut i64) -> c_int;
    pub fn exg_world_stream(world: exg_world_t, stream_out: *mut *mut c_void) -> c_int;
    pub fn exg_world_phase_cycles(w: exg_world_t, out: *mut i64) -> c_int;
    pub fn exg_world_island_count(w: exg_world_t, world: i32, n_islands: *mut i32) -> c_int;
    pub fn exg_world_island_structure(w: exg_world_t, world: i32, island: i32, kind: i32, out: *mut i32, cap: i32, len: *mut i32) -> c_int;
    pub fn exg_world_energy(w: exg_world_t, out: *mut f64) -> c_int;
    pub fn exg_storage_create(dev: exg_device_t, elem_bytes: i64, capacity: i64, out: *mut exg_storage_t) -> c_int;
    pub fn exg_storage_destroy(st: exg_storage_t) -> c_int;
    pub fn exg_slot_alloc(st: exg_storage_t, value: *const c_void, key: *mut exg_slot_key_t) -> c_int;
    pub fn exg_slot_free(st: exg_storage_t, key: exg_slot_key_t) -> c_int;
    pub fn exg_slot_read(st: exg_storage_t, key: exg_slot_key_t, out: *mut c_void) -> c_int;
    pub fn exg_slot_write(st: exg_storage_t, key: exg_slot_key_t, value: *const c_void) -> c_int;
    pub fn exg_slot_read_n(st: exg_storage_t, keys: *const exg_slot_key_t, n: i32, out: *mut c_void) -> c_int;
    pub fn exg_slot_write_n(st: exg_storage_t, keys: *const exg_slot_key_t, n: i32, values: *const c_void) -> c_int;
    pub fn exg_storage_info(st: exg_storage_t, out: *mut exg_storage_info_t) -> c_int;
    pub fn exg_ledger_check(slots: *const i32, n: i64, n_slots: i64, first_clash: *mut i64) -> c_int;
    pub fn exg_motor_exp(twist: *const f64, dt: f64, out: *mut f64) -> c_int;
    pub fn exg_motor_compose(a: *const f64, b: *const f64, out: *mut f64) -> c_int;
    pub fn exg_motor_inverse(a: *const f64, out: *mut f64) -> c_int;
    pub fn exg_motor_apply_point(m: *const f64, p: *const f64, out: *mut f64) -> c_int;
    pub fn exg_screw_transport(s: *const f64, m: *const f64, covariant: i32, out: *mut f64) -> c_int;
    pub fn exg_motor_exp_n(count: i64, twists: *const f64, dt: f64, out: *mut f64) -> c_int;
    pub fn exg_motor_compose_n(count: i64, a: *const f64, b: *const f64, out: *mut f64) -> c_int;
    pub fn exg_eval_joints(dev: exg_device_t, d_joints: *const exg_joint_t, n_joints: i32, d_pose: *const f64, d_vel: *const f64, dt: f64, warp: f64, jacobian: i32, d_out: *mut f64) -> c_int;
    pub fn exg_pivot_inverse(dev: exg_device_t, d_blocks: *const f64, n: i32, precision: i32, form: i32, warm: i32, d_out: *mut f64, d_steps: *mut i32) -> c_int;
    pub fn exg_gravity_forces(dev: exg_device_t, d_pos_mass: *const f64, d_size: *const f64, n: i32, law: i32, G: f64, softening: f64, precision: i32, d_force: *mut f64) -> c_int;
    pub fn exg_gravity_forces_noalloc(dev: exg_device_t, d_pos_mass: *const f64, d_size: *const f64, n: i32, law: i32, G: f64, softening: f64, precision: i32, d_force: *mut f64) -> c_int;
}
