"""numpy mirrors of the record layouts declared in include/exg.h.

The host-side arrays built with these dtypes are passed by pointer to the C ABI; their
byte layout must equal the C structs (checked against the library at load time).
"""
import numpy as np

BODY_DTYPE = np.dtype(
    [
        ("pose", "<f8", (8,)),
        ("momentum", "<f8", (6,)),
        ("mass", "<f8"),
        ("inertia", "<f8", (9,)),
        ("size", "<f8"),
        ("kinematic", "<i4"),
        ("diagonal", "<i4"),
    ],
    align=True,
)

JOINT_DTYPE = np.dtype(
    [("law", "<i4"), ("a", "<i4"), ("b", "<i4"), ("reserved", "<i4"), ("params", "<f8", (10,))],
    align=True,
)


STEP_PARAMS_DTYPE = np.dtype(
    [
        ("integrator", "<i4"),
        ("gravity_law", "<i4"),
        ("precision", "<i4"),
        ("newton_flags", "<i4"),
        ("G", "<f8"),
        ("softening", "<f8"),
        ("dt", "<f8"),
        ("warp", "<f8"),
        ("tol", "<f8"),
        ("max_newton", "<i4"),
        ("reserved1", "<i4"),
        ("field_accel", "<f8", (3,)),
    ],
    align=True,
)

WORLD_STATS_DTYPE = np.dtype(
    [
        ("steps", "<i8"),
        ("last_spans", "<i4"),
        ("last_newton_iterations", "<i4"),
        ("max_depth_reached", "<i4"),
        ("fatal", "<i4"),
        ("last_residual", "<f8"),
    ],
    align=True,
)

POOL_CONFIG_DTYPE = np.dtype(
    [("max_bodies", "<i8"), ("max_joints", "<i8"), ("max_worlds", "<i4"), ("precision", "<i4")], align=True
)

POOL_USAGE_DTYPE = np.dtype(
    [("worlds_used", "<i4"), ("worlds_capacity", "<i4"), ("largest_free_bodies", "<i8"),
     ("largest_free_joints", "<i8")],
    align=True,
)

SERVER_CONFIG_DTYPE = np.dtype(
    [("hbm_budget_bytes", "<i8"), ("max_bodies", "<i8"), ("max_joints", "<i8"), ("max_worlds", "<i4"),
     ("precision", "<i4"), ("steps_per_tick", "<i4"), ("pools", "<i4")],
    align=True,
)

REQUEST_INFO_DTYPE = np.dtype(
    [("steps", "<i8"), ("n_bodies", "<i4"), ("status", "<i4"), ("queued_s", "<f8"), ("latency_s", "<f8")], align=True
)

SERVER_STATS_DTYPE = np.dtype(
    [("submitted", "<i8"), ("completed", "<i8"), ("failed", "<i8"), ("ticks", "<i8"), ("steps_launched", "<i8"),
     ("body_steps", "<i8"), ("queued", "<i4"), ("running", "<i4"), ("peak_running", "<i4"), ("reserved", "<i4"),
     ("resident_bytes", "<i8"), ("peak_resident_bytes", "<i8"), ("busy_s", "<f8"), ("elapsed_s", "<f8"),
     ("p50_latency_s", "<f8"), ("p99_latency_s", "<f8"), ("mean_latency_s", "<f8")],
    align=True,
)

PENDING = 1

# Law ids and names (crates/newton/src/accelerator/mod.rs:118-132).
LAW_NAMES = ("SimpleSpringDamper", "CriticallyDampedWarped", "PerpendicularDamperWarped", "TorsionalDamperWarped")
LAW_N_PARAMS = (10, 10, 2, 1)

EXPLICIT_EULER, SYMPLECTIC_EULER, LIE_EULER, NEWTON = 0, 1, 2, 3
GRAVITY_OFF, GRAVITY_SIZE_CORE, GRAVITY_PLUMMER = 0, 1, 2
PRECISION_F64, PRECISION_MIXED, PRECISION_MIXED_FAST = 0, 1, 2


NEWTON_EXACT_POSE_FACTOR = 1
NEWTON_NS_PIVOT = 2  # mixed path: Newton-Schulz pivot inverses (warm-started, FP32 steps, FP64 correction)


def step_params(integrator=LIE_EULER, gravity_law=GRAVITY_OFF, precision=PRECISION_F64, G=1.0, softening=0.0,
                dt=1e-2, warp=1.0, tol=1e-4, max_newton=32, exact_jacobian=False, field=(0.0, 0.0, 0.0),
                ns_pivot=False):
    p = np.zeros((), dtype=STEP_PARAMS_DTYPE)
    p["newton_flags"] = (NEWTON_EXACT_POSE_FACTOR if exact_jacobian else 0) | (NEWTON_NS_PIVOT if ns_pivot else 0)
    p["integrator"] = integrator
    p["gravity_law"] = gravity_law
    p["precision"] = precision
    p["G"] = G
    p["softening"] = softening
    p["dt"] = dt
    p["warp"] = warp
    p["tol"] = tol
    p["max_newton"] = max_newton
    p["field_accel"] = field
    return p
