/* Prints sizeof and field offsets of the C ABI's records, one "type field offset" line each, so
 * the Python dtypes can be checked against the compiler's layout of include/exg.h. */
#include <stddef.h>
#include <stdio.h>
#include "exg.h"

#define SZ(T) printf(#T " sizeof %zu\n", sizeof(T))
#define OFF(T, f) printf(#T " " #f " %zu\n", offsetof(T, f))

int main(void) {
  SZ(exg_body_t); OFF(exg_body_t, pose); OFF(exg_body_t, momentum); OFF(exg_body_t, mass); OFF(exg_body_t, inertia);
  OFF(exg_body_t, size); OFF(exg_body_t, kinematic); OFF(exg_body_t, diagonal);
  SZ(exg_joint_t); OFF(exg_joint_t, law); OFF(exg_joint_t, a); OFF(exg_joint_t, b); OFF(exg_joint_t, params);
  SZ(exg_step_params_t); OFF(exg_step_params_t, integrator); OFF(exg_step_params_t, gravity_law);
  OFF(exg_step_params_t, precision); OFF(exg_step_params_t, newton_flags); OFF(exg_step_params_t, G);
  OFF(exg_step_params_t, softening); OFF(exg_step_params_t, dt); OFF(exg_step_params_t, warp);
  OFF(exg_step_params_t, tol); OFF(exg_step_params_t, max_newton); OFF(exg_step_params_t, field_accel);
  SZ(exg_world_stats_t); OFF(exg_world_stats_t, steps); OFF(exg_world_stats_t, last_spans);
  OFF(exg_world_stats_t, last_newton_iterations); OFF(exg_world_stats_t, max_depth_reached);
  OFF(exg_world_stats_t, fatal); OFF(exg_world_stats_t, last_residual);
  SZ(exg_pool_config_t); OFF(exg_pool_config_t, max_bodies); OFF(exg_pool_config_t, max_joints);
  OFF(exg_pool_config_t, max_worlds); OFF(exg_pool_config_t, precision);
  SZ(exg_pool_usage_t); OFF(exg_pool_usage_t, worlds_used); OFF(exg_pool_usage_t, worlds_capacity);
  OFF(exg_pool_usage_t, largest_free_bodies); OFF(exg_pool_usage_t, largest_free_joints);
  SZ(exg_server_config_t); OFF(exg_server_config_t, hbm_budget_bytes); OFF(exg_server_config_t, max_bodies);
  OFF(exg_server_config_t, max_joints); OFF(exg_server_config_t, max_worlds); OFF(exg_server_config_t, precision);
  OFF(exg_server_config_t, steps_per_tick);
  SZ(exg_request_info_t); OFF(exg_request_info_t, steps); OFF(exg_request_info_t, n_bodies);
  OFF(exg_request_info_t, status); OFF(exg_request_info_t, queued_s); OFF(exg_request_info_t, latency_s);
  SZ(exg_server_stats_t); OFF(exg_server_stats_t, submitted); OFF(exg_server_stats_t, completed);
  OFF(exg_server_stats_t, failed); OFF(exg_server_stats_t, ticks); OFF(exg_server_stats_t, steps_launched);
  OFF(exg_server_stats_t, body_steps); OFF(exg_server_stats_t, queued); OFF(exg_server_stats_t, running);
  OFF(exg_server_stats_t, peak_running); OFF(exg_server_stats_t, resident_bytes);
  OFF(exg_server_stats_t, peak_resident_bytes); OFF(exg_server_stats_t, busy_s); OFF(exg_server_stats_t, elapsed_s);
  OFF(exg_server_stats_t, p50_latency_s); OFF(exg_server_stats_t, p99_latency_s); OFF(exg_server_stats_t, mean_latency_s);
  return 0;
}
