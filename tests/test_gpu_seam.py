"""The precision seam at large world offsets (restating crates/newton/tests/precision_seam.rs).

The reference keeps each island's poses local to a high-precision anchor re-bound to its centre of
mass, so translating a mechanism far from the origin changes no kernel input. Here poses are
stored as absolute FP64 motors, and every Newton step works in a frame anchored at the island's
centre of mass rounded to a multiple of 1024 (the anchor carrier is FP64): a chain of five unit
masses on springs (k = 50, under a uniform field, the reference's GRID geometry: spacing 64,
non-uniform transverse velocities) translated by 2^10, 2^20 and 2^30 on every axis (multiples of
the grid, so it sits in its frame as at the origin) keeps its shape to within 64 FP64 spacings at
the offset, the rounding of the stored poses. The mixed path evaluates its FP32 Jacobian slices from
the frame's local poses, so the same holds there (plus 1e-6 for its FP32 slices' effect on the
converged iterate).
"""
import numpy as np
import pytest

from exgame_b200 import _lib, motors_np
from exgame_b200.abi import BODY_DTYPE, GRAVITY_OFF, JOINT_DTYPE, NEWTON, PRECISION_MIXED, step_params

pytestmark = pytest.mark.gpu

N, STEPS, DT = 5, 20, 1.0 / 60.0


def grid_chain(offset, h=64.0):
    """The reference's chain (precision_seam.rs:82-125): unit masses at offset + (i h, 0, 0) on
    every axis, velocities (0.02 h i, +-0.15 h (i + 1), 0.05 h i), SimpleSpringDamper k = 50,
    c = 0.1 * 2 sqrt(k m / 2), rest h between neighbours, a uniform field of -9.81 along z."""
    b = np.zeros(N, dtype=BODY_DTYPE)
    tw = np.zeros((N, 6))
    for i in range(N):
        tw[i, :3] = (offset + i * h, offset, offset)
        sign = 1.0 if i % 2 == 0 else -1.0
        b[i]["momentum"][:3] = (0.02 * h * i, 0.15 * h * sign * (i + 1.0), 0.05 * h * i)
    b["pose"] = motors_np.twist_exp_n(tw, 1.0)
    b["mass"] = 1.0
    b["inertia"][:, 0] = b["inertia"][:, 4] = b["inertia"][:, 8] = 1.0
    b["diagonal"] = 1
    b["size"] = 1.0
    k = 50.0
    c = 0.1 * 2.0 * np.sqrt(k * 1.0 * 0.5)
    j = np.zeros(N - 1, dtype=JOINT_DTYPE)
    for q in range(N - 1):
        j[q]["law"], j[q]["a"], j[q]["b"] = 0, q, q + 1
        j[q]["params"][6:10] = (h, k, c, 1e-6)
    return b, j


def relative_positions(device, offset, precision, wave=False):
    b, j = grid_chain(offset)
    p = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=DT, tol=1e-10,
                    field=(0.0, 0.0, -9.81))
    w = _lib.DeviceWorld(device, b, j, p)
    if wave:
        w.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 1)
    w.step(STEPS)
    if wave:
        assert w.get_option(_lib.DeviceWorld.OPT_LAST_WAVE_ROUNDS) > 0
    out = w.bodies()
    assert w.stats()["fatal"] == 0
    w.close()
    pos = motors_np.apply_point_n(out["pose"], np.zeros((N, 3)))
    return pos - pos[0]


@pytest.mark.parametrize("wave", [False, True])
@pytest.mark.parametrize("offset", [2.0 ** 10, 2.0 ** 20, 2.0 ** 30])
def test_far_offset_keeps_the_shape_fp64(device, offset, wave):
    ref = relative_positions(device, 0.0, 0, wave)
    far = relative_positions(device, offset, 0, wave)
    div = np.abs(far - ref).max()
    ulp = np.spacing(offset)  # FP64 spacing at the offset: positions are rounded to it
    print(f"FP64 offset {offset:.0e} ({'wave' if wave else 'island kernel'}): relative divergence {div:.3e} "
          f"(FP64 ulp {ulp:.1e})")
    assert div <= 64.0 * ulp, (div, ulp)


@pytest.mark.parametrize("offset", [2.0 ** 10, 2.0 ** 20, 2.0 ** 30])
def test_far_offset_keeps_the_shape_mixed(device, offset):
    ref = relative_positions(device, 0.0, PRECISION_MIXED)
    far = relative_positions(device, offset, PRECISION_MIXED)
    div = np.abs(far - ref).max()
    print(f"MIXED offset {offset:.0e}: relative divergence {div:.3e}")
    assert div <= 64.0 * np.spacing(offset) + 1e-6, div
