"""ctypes binding of the oracle (oracle/_build/liboracle.so) for the test suite and the bench's
CPU-baseline leg. The oracle is the checker, never the thing measured or shipped."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_L = None
_dp = ctypes.POINTER(ctypes.c_double)


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return LIB


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_world_create.restype = ctypes.c_void_p
        L.orc_world_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_world_destroy.argtypes = [ctypes.c_void_p]
        L.orc_world_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_worlds_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_world_get_bodies.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_world_set_state.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_world_set_epoch.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.orc_world_energy.restype = ctypes.c_double
        L.orc_world_energy.argtypes = [ctypes.c_void_p]
        L.orc_world_island_count.argtypes = [ctypes.c_void_p]
        L.orc_world_island_structure.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.c_int]
        L.orc_world_island_stats.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int)]
        L.orc_power.restype = ctypes.c_double
        L.orc_pair_force_literal.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_void_p]
        L.orc_twist_exp.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        for fn in ("orc_plain_eval", "orc_jacobian_eval"):
            getattr(L, fn).argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
        L.orc_gravity_forces.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_void_p]
        L.orc_body_post.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4 + [ctypes.c_double, ctypes.c_double] + \
            [ctypes.c_void_p] * 3
        L.orc_study_forms.argtypes = [ctypes.c_double, ctypes.c_void_p]
        L.orc_study_forms_f32.argtypes = [ctypes.c_float, ctypes.c_void_p]
        _L = L
    return _L


def p(a):
    # data_as keeps a reference to the array, so temporaries outlive the call
    return a.ctypes.data_as(ctypes.c_void_p)


def arr(x):
    return np.ascontiguousarray(x, dtype=np.float64)


class OracleWorld:
    SOLVER_EXACT, SOLVER_REFERENCE_NS = 0, 1

    def __init__(self, bodies, joints, params, solver=0, ns_warm=2, ns_seed=24):
        self._b = np.ascontiguousarray(bodies)
        self._j = np.ascontiguousarray(joints)
        self._p = np.ascontiguousarray(params).reshape(())
        self.h = lib().orc_world_create(p(self._b), len(self._b), p(self._j), len(self._j), p(self._p), solver,
                                        ns_warm, ns_seed)
        self.n = len(self._b)

    def step(self, n=1):
        lib().orc_world_step(self.h, int(n))

    def bodies(self):
        out = np.zeros_like(self._b)
        lib().orc_world_get_bodies(self.h, p(out))
        return out

    def set_state(self, bodies):
        """Overwrite every body's pose and momentum from records (the islands stay)."""
        b = np.ascontiguousarray(bodies)
        assert len(b) == self.n
        lib().orc_world_set_state(self.h, p(b))

    def energy(self):
        return lib().orc_world_energy(self.h)

    def set_epoch(self, dt, warp=1.0):
        """dt and warp of the following steps (a variable frame time); the islands stay."""
        lib().orc_world_set_epoch(self.h, float(dt), float(warp))

    def island_stats(self):
        out = []
        for k in range(lib().orc_world_island_count(self.h)):
            s, it = ctypes.c_int(), ctypes.c_int()
            lib().orc_world_island_stats(self.h, k, ctypes.byref(s), ctypes.byref(it))
            out.append((s.value, it.value))
        return out

    STRUCT_KINDS = {"bodies": 1, "joint_ends": 2, "order": 3, "incidence_ptr": 4, "incidence": 5, "joints": 7}

    def island_count(self):
        return lib().orc_world_island_count(self.h)

    def island_structure(self, island, kind):
        """The oracle's restatement of one island map (islands, order, bake_incidence)."""
        cap = 8 * (len(self._b) + 3 * len(self._j)) + 8
        out = np.zeros(cap, dtype=np.int32)
        n = lib().orc_world_island_structure(self.h, int(island), self.STRUCT_KINDS[kind], p(out), cap)
        assert n >= 0
        out = out[:n]
        return out.reshape(-1, 3) if kind == "joint_ends" else out

    def __del__(self):
        try:
            lib().orc_world_destroy(self.h)
        except Exception:
            pass


def worlds_step(worlds, steps):
    """Step independent oracle worlds `steps` times, spread over the oracle's threads (OpenMP)."""
    hs = (ctypes.c_void_p * len(worlds))(*[w.h for w in worlds])
    lib().orc_worlds_step(hs, len(worlds), int(steps))


def twist_exp(t, dt=1.0):
    o = np.zeros(8)
    lib().orc_twist_exp(p(arr(t)), float(dt), p(o))
    return o


def plain_eval(law, params, pa, pb, va, vb, dt, warp):
    o = np.zeros(12)
    lib().orc_plain_eval(int(law), p(arr(params)), p(arr(pa)), p(arr(pb)), p(arr(va)), p(arr(vb)), float(dt),
                         float(warp), p(o))
    return o


def jacobian_eval(law, params, pa, pb, va, vb, dt, warp):
    o = np.zeros(300)
    lib().orc_jacobian_eval(int(law), p(arr(params)), p(arr(pa)), p(arr(pb)), p(arr(va)), p(arr(vb)), float(dt),
                            float(warp), p(o))
    return o.reshape(12, 25)


def gravity_forces(bodies, law, G, eps):
    b = np.ascontiguousarray(bodies)
    o = np.zeros((len(b), 3))
    lib().orc_gravity_forces(p(b), len(b), int(law), float(G), float(eps), p(o))
    return o
