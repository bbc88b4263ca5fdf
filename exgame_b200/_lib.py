"""ctypes binding of libexg.so (include/exg.h).

The library is built in-tree (exgame_b200/libexg.so). Loading fails loudly when it is missing:
there is no CPU fallback for the compute path.
"""
import ctypes
import os
import weakref

import numpy as np

from .abi import (BODY_DTYPE, JOINT_DTYPE, PENDING, POOL_CONFIG_DTYPE, POOL_USAGE_DTYPE, PRECISION_F64,
                  REQUEST_INFO_DTYPE, SERVER_CONFIG_DTYPE, SERVER_STATS_DTYPE, STEP_PARAMS_DTYPE, WORLD_STATS_DTYPE)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libexg.so")

EXG_OK = 0
STATUS_NAMES = {
    0: "EXG_OK", -1: "EXG_ERR_NO_SHADER", -2: "EXG_ERR_TRAP", -3: "EXG_ERR_FATAL", -4: "EXG_ERR_WORKER_GONE",
    -5: "EXG_ERR_BACKEND", -10: "EXG_ERR_EPOCH_IN_PROGRESS", -11: "EXG_ERR_ALREADY_OWNED",
    -12: "EXG_ERR_FOREIGN_ACCELERATOR", -13: "EXG_ERR_DUPLICATE_MECHANISM", -20: "EXG_ERR_INVALID_ARGUMENT",
    -21: "EXG_ERR_OUT_OF_MEMORY", -22: "EXG_ERR_UNSUPPORTED", -23: "EXG_ERR_TIMEOUT", -24: "EXG_ERR_NO_DEVICE",
}

_c_double_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

# name -> (restype, argtypes); every symbol declared in include/exg.h
SIGNATURES = {
    "exg_abi_version": (ctypes.c_int, []),
    "exg_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "exg_device_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(_vp)]),
    "exg_device_destroy": (ctypes.c_int, [_vp]),
    "exg_device_synchronize": (ctypes.c_int, [_vp]),
    "exg_device_kernel_launches": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "exg_device_stream": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "exg_device_profile": (ctypes.c_int, [_vp, ctypes.c_int32]),
    "exg_device_profile_read": (ctypes.c_int, [_vp, ctypes.c_int32, _c_double_p, ctypes.POINTER(ctypes.c_int64)]),
    "exg_device_set_tuning": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32]),
    "exg_device_get_tuning": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "exg_law_lookup": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    "exg_world_create": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp, ctypes.c_int32, _vp, ctypes.POINTER(_vp)]),
    "exg_world_destroy": (ctypes.c_int, [_vp]),
    "exg_world_step": (ctypes.c_int, [_vp, ctypes.c_int32]),
    "exg_world_get_bodies": (ctypes.c_int, [_vp, _vp, ctypes.c_int32]),
    "exg_world_set_bodies": (ctypes.c_int, [_vp, _vp, ctypes.c_int32]),
    "exg_world_get_state": (ctypes.c_int, [_vp, _vp, ctypes.c_int32]),
    "exg_batch_set_joints": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, ctypes.c_int32]),
    "exg_world_stream": (ctypes.c_int, [_vp, _vp]),
    "exg_world_set_state": (ctypes.c_int, [_vp, _vp, ctypes.c_int32]),
    "exg_world_stats": (ctypes.c_int, [_vp, _vp]),
    "exg_world_energy": (ctypes.c_int, [_vp, _c_double_p]),
    "exg_batch_create": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "exg_batch_get_world": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, ctypes.c_int32]),
    "exg_batch_set_world": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, ctypes.c_int32]),
    "exg_batch_world_stats": (ctypes.c_int, [_vp, ctypes.c_int32, _vp]),
    "exg_pool_create": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
    "exg_pool_admit": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp, ctypes.c_int32, _vp,
                                      ctypes.POINTER(ctypes.c_int32)]),
    "exg_pool_release": (ctypes.c_int, [_vp, ctypes.c_int32]),
    "exg_pool_free": (ctypes.c_int, [_vp, _vp]),
    "exg_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "exg_host_free": (ctypes.c_int, [_vp]),
    "exg_world_footprint": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _vp, ctypes.POINTER(ctypes.c_int64)]),
    "exg_server_create": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
    "exg_server_submit": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp, ctypes.c_int32, _vp, ctypes.c_int32,
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "exg_server_poll": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp, ctypes.c_int32, _vp]),
    "exg_server_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_int32, _vp, ctypes.c_int32, _vp]),
    "exg_server_stats": (ctypes.c_int, [_vp, _vp]),
    "exg_server_reset_stats": (ctypes.c_int, [_vp]),
    "exg_server_destroy": (ctypes.c_int, [_vp]),
    "exg_world_set_option": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int64]),
    "exg_world_get_option": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int64)]),
    "exg_pool_set_steps": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32]),
    "exg_pool_steps_left": (ctypes.c_int, [_vp, _vp, ctypes.c_int32]),
    "exg_world_phase_cycles": (ctypes.c_int, [_vp, _vp]),
    "exg_world_island_count": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "exg_batch_set_epoch": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_double, ctypes.c_double]),
    "exg_storage_create": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(_vp)]),
    "exg_storage_destroy": (ctypes.c_int, [_vp]),
    "exg_slot_alloc": (ctypes.c_int, [_vp, _vp, _vp]),
    "exg_slot_free": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "exg_slot_read": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp]),
    "exg_slot_write": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp]),
    "exg_slot_read_n": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp]),
    "exg_slot_write_n": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp]),
    "exg_storage_info": (ctypes.c_int, [_vp, _vp]),
    "exg_ledger_check": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "exg_world_island_structure": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp,
                                                  ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "exg_motor_exp": (ctypes.c_int, [_vp, ctypes.c_double, _vp]),
    "exg_motor_compose": (ctypes.c_int, [_vp, _vp, _vp]),
    "exg_motor_inverse": (ctypes.c_int, [_vp, _vp]),
    "exg_motor_apply_point": (ctypes.c_int, [_vp, _vp, _vp]),
    "exg_screw_transport": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp]),
    "exg_motor_exp_n": (ctypes.c_int, [ctypes.c_int64, _vp, ctypes.c_double, _vp]),
    "exg_motor_compose_n": (ctypes.c_int, [ctypes.c_int64, _vp, _vp, _vp]),
    "exg_eval_joints": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int32, _vp]),
    "exg_pivot_inverse": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp, _vp]),
    "exg_gravity_forces": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int32, _vp]),
    "exg_gravity_forces_noalloc": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_int32, _vp]),
}


class ExgError(RuntimeError):
    """A non-zero status from the C ABI (EvalError / StructureError of the reference)."""

    def __init__(self, status, where=""):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        msg = lib().exg_status_string(status).decode() if _LIB is not None else ""
        super().__init__(f"{where}: {self.name} ({msg})" if where else f"{self.name} ({msg})")


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libexg.so is not built ({LIB_PATH}); run `python -m exgame_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status, where=""):
    if status != EXG_OK:
        raise ExgError(status, where)


def ptr(a):
    # data_as keeps a reference to the array, so temporaries outlive the call
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else ctypes.c_void_p(0)


def motor_exp(twist, dt=1.0):
    t = np.ascontiguousarray(twist, dtype=np.float64)
    out = np.zeros(8)
    check(lib().exg_motor_exp(ptr(t), float(dt), ptr(out)), "exg_motor_exp")
    return out


def motor_compose(a, b):
    """'first a, then b' (Motor::compose)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros(8)
    check(lib().exg_motor_compose(ptr(a), ptr(b), ptr(out)), "exg_motor_compose")
    return out


def motor_exp_n(twists, dt=1.0):
    t = np.ascontiguousarray(twists, dtype=np.float64).reshape(-1, 6)
    out = np.zeros((len(t), 8))
    check(lib().exg_motor_exp_n(len(t), ptr(t), float(dt), ptr(out)), "exg_motor_exp_n")
    return out


def motor_compose_n(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 8)
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, 8)
    out = np.zeros((len(a), 8))
    check(lib().exg_motor_compose_n(len(a), ptr(a), ptr(b), ptr(out)), "exg_motor_compose_n")
    return out


def motor_inverse(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.zeros(8)
    check(lib().exg_motor_inverse(ptr(a), ptr(out)), "exg_motor_inverse")
    return out


def motor_apply_point(m, p):
    m = np.ascontiguousarray(m, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    out = np.zeros(3)
    check(lib().exg_motor_apply_point(ptr(m), ptr(p), ptr(out)), "exg_motor_apply_point")
    return out


def screw_transport(s, m, covariant):
    s = np.ascontiguousarray(s, dtype=np.float64)
    m = np.ascontiguousarray(m, dtype=np.float64)
    out = np.zeros(6)
    check(lib().exg_screw_transport(ptr(s), ptr(m), int(covariant), ptr(out)), "exg_screw_transport")
    return out


def law_lookup(name):
    law = ctypes.c_int32()
    n = ctypes.c_int32()
    check(lib().exg_law_lookup(name.encode(), ctypes.byref(law), ctypes.byref(n)), f"exg_law_lookup({name})")
    return law.value, n.value


class Device:
    """A CUDA device context (replaces the reference's GpuAccelerator::new)."""

    def __init__(self, ordinal=0):
        h = ctypes.c_void_p()
        check(lib().exg_device_create(int(ordinal), ctypes.byref(h)), "exg_device_create")
        self.handle = h
        self.ordinal = ordinal
        self._owned = weakref.WeakSet()  # worlds, pools and servers made on this device

    def kernel_launches(self):
        v = ctypes.c_uint64()
        check(lib().exg_device_kernel_launches(self.handle, ctypes.byref(v)))
        return v.value

    def synchronize(self):
        check(lib().exg_device_synchronize(self.handle))

    def stream(self):
        s = ctypes.c_void_p()
        check(lib().exg_device_stream(self.handle, ctypes.byref(s)))
        return s.value

    TUNE_GRAVITY_CTAS_PER_SM, TUNE_WAVE_BLOCKS_PER_SM, TUNE_WAVE_MIN_BODIES, TUNE_WAVE_NARROW_LEVEL = 1, 2, 3, 4

    def set_tuning(self, key, value):
        check(lib().exg_device_set_tuning(self.handle, int(key), int(value)), "exg_device_set_tuning")

    def get_tuning(self, key):
        v = ctypes.c_int32()
        check(lib().exg_device_get_tuning(self.handle, int(key), ctypes.byref(v)), "exg_device_get_tuning")
        return v.value

    def profile(self, enable):
        check(lib().exg_device_profile(self.handle, int(bool(enable))))

    PROF_GRAVITY, PROF_JOINTS, PROF_INTEGRATE, PROF_NEWTON, PROF_BODY_PRE, PROF_NEWTON_WAVE = 0, 1, 2, 3, 4, 5

    def profile_read(self, kind):
        ms, n = ctypes.c_double(), ctypes.c_int64()
        check(lib().exg_device_profile_read(self.handle, int(kind), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def close(self):
        """Destroy the device; the worlds, pools and servers made on it are closed first (the
        library refuses to destroy a device under live handles)."""
        if self.handle:
            for h in list(self._owned):
                h.close()
            lib().exg_device_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceWorld:
    """A device-resident world of bodies and joints stepped by the CUDA path."""

    def __init__(self, device, bodies, joints, params):
        self.device = device
        self.bodies_host = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        self.joints_host = np.ascontiguousarray(joints, dtype=JOINT_DTYPE)
        self.params = np.ascontiguousarray(params, dtype=STEP_PARAMS_DTYPE).reshape(())
        h = ctypes.c_void_p()
        check(lib().exg_world_create(device.handle, ptr(self.bodies_host), len(self.bodies_host), ptr(self.joints_host),
                                     len(self.joints_host), ptr(self.params), ctypes.byref(h)), "exg_world_create")
        self.handle = h
        device._owned.add(self)
        self.n = len(self.bodies_host)

    def step(self, n_steps=1):
        check(lib().exg_world_step(self.handle, int(n_steps)), "exg_world_step")

    def bodies(self, out=None):
        """Every body of the handle (into `out` when given, e.g. a host_bodies buffer)."""
        if out is None:
            out = np.zeros(self.n, dtype=BODY_DTYPE)
        if out.dtype != BODY_DTYPE or len(out) != self.n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous BODY_DTYPE array of the handle's body count")
        check(lib().exg_world_get_bodies(self.handle, ptr(out), self.n), "exg_world_get_bodies")
        return out

    def set_bodies(self, bodies):
        b = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        check(lib().exg_world_set_bodies(self.handle, ptr(b), len(b)), "exg_world_set_bodies")

    def state(self, out=None):
        """Every body's (pose[8], momentum[6]) as an (n, 14) array (into `out` when given, e.g. a
        host_state buffer)."""
        if out is None:
            out = np.zeros((self.n, 14), dtype=np.float64)
        if out.dtype != np.float64 or out.shape != (self.n, 14) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of shape (n_bodies, 14)")
        check(lib().exg_world_get_state(self.handle, ptr(out), self.n), "exg_world_get_state")
        return out

    def set_joints(self, joints, world=0):
        """Replace the joints of `world` (0 for a single world; a batch index or pool slot)."""
        j = np.ascontiguousarray(joints, dtype=JOINT_DTYPE)
        check(lib().exg_batch_set_joints(self.handle, int(world), ptr(j), len(j)), "exg_batch_set_joints")

    def set_epoch(self, dt, warp=1.0, world=0):
        """dt and warp of `world` for the following steps (Epoch::standalone(dt, warp))."""
        check(lib().exg_batch_set_epoch(self.handle, int(world), float(dt), float(warp)), "exg_batch_set_epoch")

    def set_state(self, state):
        st = np.ascontiguousarray(state, dtype=np.float64)
        if st.shape != (self.n, 14):
            raise ValueError("state must have shape (n_bodies, 14)")
        check(lib().exg_world_set_state(self.handle, ptr(st), self.n), "exg_world_set_state")

    def stats(self):
        s = np.zeros((), dtype=WORLD_STATS_DTYPE)
        check(lib().exg_world_stats(self.handle, ptr(s)), "exg_world_stats")
        return s

    OPT_WAVE_MIN_BODIES, OPT_WAVE_MAX_LEVELS, OPT_LAST_WAVE_ROUNDS, OPT_WAVE_HOST_ROUNDS, OPT_OWN_STREAM = 1, 2, 3, 4, 5
    OPT_WAVE_LEVEL_MAX_WIDTH, OPT_WAVE_LEVEL_MIN_WIDTH = 6, 7

    def stream(self):
        """The CUDA stream (as an integer handle) this world's work runs on."""
        s = ctypes.c_void_p()
        check(lib().exg_world_stream(self.handle, ctypes.byref(s)), "exg_world_stream")
        return s.value

    def set_option(self, option, value):
        check(lib().exg_world_set_option(self.handle, int(option), int(value)), "exg_world_set_option")

    def get_option(self, option):
        v = ctypes.c_int64()
        check(lib().exg_world_get_option(self.handle, int(option), ctypes.byref(v)), "exg_world_get_option")
        return v.value

    PHASES = ("pre", "joints+jacobian", "gather+post", "assemble", "solve", "line search", "commit", "other")

    def phase_cycles(self):
        out = np.zeros(8, dtype=np.int64)
        check(lib().exg_world_phase_cycles(self.handle, ptr(out)), "exg_world_phase_cycles")
        return dict(zip(self.PHASES, out.tolist()))

    def energy(self):
        e = ctypes.c_double()
        check(lib().exg_world_energy(self.handle, ctypes.byref(e)), "exg_world_energy")
        return e.value

    STRUCT_KINDS = {"bodies": 1, "joint_ends": 2, "order": 3, "incidence_ptr": 4, "incidence": 5, "parent": 6,
                    "joints": 7}

    def island_count(self, world=0):
        n = ctypes.c_int32()
        check(lib().exg_world_island_count(self.handle, int(world), ctypes.byref(n)), "exg_world_island_count")
        return n.value

    def island_structure(self, island, kind, world=0):
        """One integer map of an implicit island's solver structure, read back from the device
        (kind: a key of STRUCT_KINDS). joint_ends comes as an (n_joints, 3) array: law, a, b."""
        k = self.STRUCT_KINDS[kind]
        n = ctypes.c_int32()
        st = lib().exg_world_island_structure(self.handle, int(world), int(island), k, None, 0, ctypes.byref(n))
        if st != EXG_OK and n.value == 0 and st != -20:
            check(st, "exg_world_island_structure")
        out = np.zeros(max(n.value, 1), dtype=np.int32)
        check(lib().exg_world_island_structure(self.handle, int(world), int(island), k, ptr(out), len(out),
                                               ctypes.byref(n)), "exg_world_island_structure")
        out = out[:n.value]
        return out.reshape(-1, 3) if kind == "joint_ends" else out

    def close(self):
        if self.handle:
            lib().exg_world_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceBatch(DeviceWorld):
    """Many independent worlds of uneven size stepped together by one set of launches per step."""

    def __init__(self, device, worlds):
        """worlds: list of (bodies, joints, params); joint body indices local to their world."""
        self.device = device
        self.counts = np.array([len(b) for b, _, _ in worlds], dtype=np.int32)
        self.jcounts = np.array([len(j) for _, j, _ in worlds], dtype=np.int32)
        self.bodies_host = np.ascontiguousarray(np.concatenate([b for b, _, _ in worlds]), dtype=BODY_DTYPE)
        js = [j for _, j, _ in worlds if len(j)]
        self.joints_host = np.ascontiguousarray(np.concatenate(js) if js else np.zeros(0, JOINT_DTYPE), dtype=JOINT_DTYPE)
        self.params = np.ascontiguousarray(np.array([p for _, _, p in worlds], dtype=STEP_PARAMS_DTYPE))
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        h = ctypes.c_void_p()
        check(lib().exg_batch_create(device.handle, len(worlds), ptr(self.counts), ptr(self.jcounts),
                                     ptr(self.bodies_host), ptr(self.joints_host), ptr(self.params), ctypes.byref(h)),
              "exg_batch_create")
        self.handle = h
        device._owned.add(self)
        self.n = int(self.counts.sum())
        self.n_worlds = len(worlds)

    def world_bodies(self, k):
        out = np.zeros(int(self.counts[k]), dtype=BODY_DTYPE)
        check(lib().exg_batch_get_world(self.handle, int(k), ptr(out), len(out)), "exg_batch_get_world")
        return out

    def set_world_bodies(self, k, bodies):
        b = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        check(lib().exg_batch_set_world(self.handle, int(k), ptr(b), len(b)), "exg_batch_set_world")

    def world_stats(self, k):
        s = np.zeros((), dtype=WORLD_STATS_DTYPE)
        check(lib().exg_batch_world_stats(self.handle, int(k), ptr(s)), "exg_batch_world_stats")
        return s


class DevicePool(DeviceWorld):
    """Worlds admitted into and released from fixed-capacity device arrays; one step advances
    every admitted world. The serving form of DeviceBatch."""

    def __init__(self, device, max_bodies, max_joints, max_worlds, precision=PRECISION_F64):
        self.device = device
        cfg = np.zeros((), dtype=POOL_CONFIG_DTYPE)
        cfg["max_bodies"], cfg["max_joints"], cfg["max_worlds"], cfg["precision"] = (
            max_bodies, max_joints, max_worlds, precision)
        h = ctypes.c_void_p()
        check(lib().exg_pool_create(device.handle, ptr(cfg), ctypes.byref(h)), "exg_pool_create")
        self.handle = h
        device._owned.add(self)
        self.counts = {}  # slot -> body count

    @property
    def n(self):
        return int(sum(self.counts.values()))

    def admit(self, bodies, joints, params):
        b = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        j = np.ascontiguousarray(joints, dtype=JOINT_DTYPE)
        p = np.ascontiguousarray(params, dtype=STEP_PARAMS_DTYPE).reshape(())
        slot = ctypes.c_int32()
        check(lib().exg_pool_admit(self.handle, ptr(b), len(b), ptr(j), len(j), ptr(p), ctypes.byref(slot)),
              "exg_pool_admit")
        self.counts[slot.value] = len(b)
        return slot.value

    def release(self, slot):
        check(lib().exg_pool_release(self.handle, int(slot)), "exg_pool_release")
        del self.counts[slot]

    def set_steps(self, slot, steps):
        check(lib().exg_pool_set_steps(self.handle, int(slot), int(steps)), "exg_pool_set_steps")

    def steps_left(self, n_slots):
        out = np.zeros(int(n_slots), dtype=np.int32)
        check(lib().exg_pool_steps_left(self.handle, ptr(out), len(out)), "exg_pool_steps_left")
        return out

    def usage(self):
        u = np.zeros((), dtype=POOL_USAGE_DTYPE)
        check(lib().exg_pool_free(self.handle, ptr(u)), "exg_pool_free")
        return u

    def world_bodies(self, slot):
        out = np.zeros(self.counts[slot], dtype=BODY_DTYPE)
        check(lib().exg_batch_get_world(self.handle, int(slot), ptr(out), len(out)), "exg_batch_get_world")
        return out

    def set_world_bodies(self, slot, bodies):
        b = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        check(lib().exg_batch_set_world(self.handle, int(slot), ptr(b), len(b)), "exg_batch_set_world")

    def world_stats(self, slot):
        s = np.zeros((), dtype=WORLD_STATS_DTYPE)
        check(lib().exg_batch_world_stats(self.handle, int(slot), ptr(s)), "exg_batch_world_stats")
        return s


def host_bodies(n):
    """A zeroed BODY_DTYPE array of n records in page-locked host memory (exg_host_alloc), freed
    when the array is collected. Record copies to and from the device run at the link's rate."""
    import weakref
    nbytes = max(1, int(n) * BODY_DTYPE.itemsize)
    p = ctypes.c_void_p()
    check(lib().exg_host_alloc(nbytes, ctypes.byref(p)), "exg_host_alloc")
    buf = (ctypes.c_char * nbytes).from_address(p.value)
    arr = np.frombuffer(buf, dtype=BODY_DTYPE, count=int(n))
    arr[...] = np.zeros((), dtype=BODY_DTYPE)
    weakref.finalize(buf, lib().exg_host_free, ctypes.c_void_p(p.value))
    return arr


def host_state(n):
    """A zeroed (n, 14) float64 array in page-locked host memory, for DeviceWorld.state/set_state
    (pose[8] then momentum[6] per body)."""
    import weakref
    nbytes = max(1, int(n) * 14 * 8)
    p = ctypes.c_void_p()
    check(lib().exg_host_alloc(nbytes, ctypes.byref(p)), "exg_host_alloc")
    buf = (ctypes.c_char * nbytes).from_address(p.value)
    arr = np.frombuffer(buf, dtype=np.float64, count=int(n) * 14).reshape(int(n), 14)
    arr[...] = 0.0
    weakref.finalize(buf, lib().exg_host_free, ctypes.c_void_p(p.value))
    return arr


def world_footprint(n_bodies, n_joints, params):
    """Device bytes a world holds while admitted to a pool (exg_world_footprint)."""
    p = np.ascontiguousarray(params, dtype=STEP_PARAMS_DTYPE).reshape(())
    out = ctypes.c_int64()
    check(lib().exg_world_footprint(int(n_bodies), int(n_joints), ptr(p), ctypes.byref(out)), "exg_world_footprint")
    return out.value


class Server:
    """Continuous-batching request loop (exg_server_*): submit worlds with step counts from any
    thread; a native worker admits them into a device pool against a memory budget and steps them
    together; results come back through poll / wait."""

    def __init__(self, device, hbm_budget_bytes=150 * 10**9, max_bodies=1 << 22, max_joints=1 << 22,
                 max_worlds=4096, precision=PRECISION_F64, steps_per_tick=16, pools=2):
        self.device = device
        cfg = np.zeros((), dtype=SERVER_CONFIG_DTYPE)
        cfg["hbm_budget_bytes"], cfg["max_bodies"], cfg["max_joints"] = hbm_budget_bytes, max_bodies, max_joints
        cfg["max_worlds"], cfg["precision"], cfg["steps_per_tick"] = max_worlds, precision, steps_per_tick
        cfg["pools"] = pools
        h = ctypes.c_void_p()
        check(lib().exg_server_create(device.handle, ptr(cfg), ctypes.byref(h)), "exg_server_create")
        self.handle = h
        device._owned.add(self)
        self.sizes = {}

    def submit(self, bodies, joints, params, steps):
        b = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        j = np.ascontiguousarray(joints, dtype=JOINT_DTYPE)
        p = np.ascontiguousarray(params, dtype=STEP_PARAMS_DTYPE).reshape(())
        rid = ctypes.c_uint64()
        check(lib().exg_server_submit(self.handle, ptr(b), len(b), ptr(j), len(j), ptr(p), int(steps),
                                      ctypes.byref(rid)), "exg_server_submit")
        self.sizes[rid.value] = len(b)
        return rid.value

    def _collect(self, st, rid, out, info):
        if st == PENDING:
            return None
        self.sizes.pop(rid, None)
        check(st, "exg_server request")
        return out, info

    def poll(self, rid):
        """None while pending; (bodies, info) once done (raises ExgError if the request failed)."""
        out = np.zeros(self.sizes.get(rid, 0), dtype=BODY_DTYPE)
        info = np.zeros((), dtype=REQUEST_INFO_DTYPE)
        st = lib().exg_server_poll(self.handle, ctypes.c_uint64(rid), ptr(out), len(out), ptr(info))
        return self._collect(st, rid, out, info)

    def wait(self, rid, timeout_ms=60000):
        out = np.zeros(self.sizes.get(rid, 0), dtype=BODY_DTYPE)
        info = np.zeros((), dtype=REQUEST_INFO_DTYPE)
        st = lib().exg_server_wait(self.handle, ctypes.c_uint64(rid), int(timeout_ms), ptr(out), len(out), ptr(info))
        return self._collect(st, rid, out, info)

    def stats(self):
        s = np.zeros((), dtype=SERVER_STATS_DTYPE)
        check(lib().exg_server_stats(self.handle, ptr(s)), "exg_server_stats")
        return {k: s[k].item() for k in s.dtype.names if k != "reserved"}

    def reset_stats(self):
        check(lib().exg_server_reset_stats(self.handle), "exg_server_reset_stats")

    def close(self):
        if self.handle:
            lib().exg_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ── typed slot storage and the one-writer ledger ─────────────────────────────
SLOT_KEY_DTYPE = np.dtype([("index", np.uint32), ("generation", np.uint32)])
STORAGE_INFO_DTYPE = np.dtype([("buffer", np.uint64), ("elem_bytes", np.int64), ("capacity", np.int64),
                               ("len", np.int64), ("live", np.int64), ("generation", np.uint64)])


def _key_word(key):
    """An exg_slot_key_t passed by value: (index, generation) packed little-endian in 64 bits."""
    k = np.asarray(key, dtype=SLOT_KEY_DTYPE).reshape(())
    return int(k["index"]) | (int(k["generation"]) << 32)


class SlotStorage:
    """Typed slot storage on the device (aristotle::World per-type storage): elements of one numpy
    dtype, keys (index, generation), lowest free slot reused, growth that keeps indices and bumps
    the storage's generation."""

    def __init__(self, device, dtype, capacity=256):
        self.device = device
        self.dtype = np.dtype(dtype)
        if self.dtype.itemsize % 4:
            raise ValueError("element size must be a multiple of 4 bytes")
        h = ctypes.c_void_p()
        check(lib().exg_storage_create(device.handle, self.dtype.itemsize, int(capacity), ctypes.byref(h)),
              "exg_storage_create")
        self.handle = h
        device._owned.add(self)

    def alloc(self, value):
        v = np.ascontiguousarray(np.asarray(value, dtype=self.dtype).reshape(()))
        key = np.zeros((), dtype=SLOT_KEY_DTYPE)
        check(lib().exg_slot_alloc(self.handle, ptr(v), ptr(key)), "exg_slot_alloc")
        return key

    def free(self, key):
        check(lib().exg_slot_free(self.handle, _key_word(key)), "exg_slot_free")

    def read(self, key):
        out = np.zeros((), dtype=self.dtype)
        check(lib().exg_slot_read(self.handle, _key_word(key), ptr(out)), "exg_slot_read")
        return out

    def write(self, key, value):
        v = np.ascontiguousarray(np.asarray(value, dtype=self.dtype).reshape(()))
        check(lib().exg_slot_write(self.handle, _key_word(key), ptr(v)), "exg_slot_write")

    def read_n(self, keys):
        k = np.ascontiguousarray(keys, dtype=SLOT_KEY_DTYPE)
        out = np.zeros(len(k), dtype=self.dtype)
        check(lib().exg_slot_read_n(self.handle, ptr(k), len(k), ptr(out)), "exg_slot_read_n")
        return out

    def write_n(self, keys, values):
        k = np.ascontiguousarray(keys, dtype=SLOT_KEY_DTYPE)
        v = np.ascontiguousarray(values, dtype=self.dtype)
        if len(v) != len(k):
            raise ValueError("one value per key")
        check(lib().exg_slot_write_n(self.handle, ptr(k), len(k), ptr(v)), "exg_slot_write_n")

    def info(self):
        out = np.zeros((), dtype=STORAGE_INFO_DTYPE)
        check(lib().exg_storage_info(self.handle, ptr(out)), "exg_storage_info")
        return out

    def close(self):
        if self.handle:
            lib().exg_storage_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ledger_check(slots, n_slots):
    """The one-writer check of a scatter map: (status, first offending position or -1)."""
    s = np.ascontiguousarray(slots, dtype=np.int32)
    clash = ctypes.c_int64()
    st = lib().exg_ledger_check(ptr(s), len(s), int(n_slots), ctypes.byref(clash))
    return st, clash.value
