"""Islands whose dynamic bodies form cycles: the reference's curtain (a grid of point bodies joined
by axial springs along both axes, the top row kinematic; crates/newton/tests/cloth_grid_stability.rs,
cloth_scaling.rs), solved on the device by block LU on a minimum-degree elimination order.

Checked against the oracle with both of its solvers: exact dense LU (SOLVER_EXACT) and the
reference's dense-block Newton-Schulz (SOLVER_REFERENCE_NS), at the cloth_scaling sizes; in mixed
precision over 1000 steps; the reference's stability cases (frame-time spikes, absurdly large steps);
and a batch mixing curtains with trees, each world bit for bit as when stepped alone."""
import numpy as np
import pytest

from exgame_b200 import _lib, motors_np, scenarios
from exgame_b200.abi import NEWTON, PRECISION_F64, PRECISION_MIXED, step_params

pytestmark = pytest.mark.gpu

SIZES = [(2, 4), (3, 6), (4, 8), (5, 10)]  # cloth_scaling.rs: (cols, rows)


def pose_rel(got, want):
    return float((np.abs(got["pose"] - want["pose"]).max(axis=1) /
                  np.maximum(1.0, np.abs(want["pose"]).max(axis=1))).max())


def mom_rel(got, want):
    return float(np.abs(got["momentum"] - want["momentum"]).max() / max(np.abs(want["momentum"]).max(), 1e-300))


@pytest.mark.parametrize("cols,rows", SIZES)
def test_cloth_scaling_sizes_match_both_oracle_solvers(device, oracle, cols, rows):
    b, j, p = scenarios.cloth_world(cols, rows, tol=1e-10)
    steps = 60
    dw = _lib.DeviceWorld(device, b, j, p)
    dw.step(steps)
    got = dw.bodies()
    assert int(dw.stats()["fatal"]) == 0
    exact = oracle.OracleWorld(b, j, p, solver=oracle.OracleWorld.SOLVER_EXACT)
    exact.step(steps)
    assert pose_rel(got, exact.bodies()) <= 1e-10 and mom_rel(got, exact.bodies()) <= 1e-8
    ns = oracle.OracleWorld(b, j, p, solver=oracle.OracleWorld.SOLVER_REFERENCE_NS)
    ns.step(steps)
    # the reference's solver converges to the same step within the Newton tolerance
    assert pose_rel(got, ns.bodies()) <= 1e-9, pose_rel(got, ns.bodies())
    dw.close()


def test_larger_cloth_matches_the_oracle(device, oracle):
    b, j, p = scenarios.cloth_world(8, 16, tol=1e-10)
    dw = _lib.DeviceWorld(device, b, j, p)
    dw.step(10)
    ow = oracle.OracleWorld(b, j, p)
    ow.step(10)
    got, want = dw.bodies(), ow.bodies()
    assert pose_rel(got, want) <= 1e-10 and mom_rel(got, want) <= 1e-8, (pose_rel(got, want), mom_rel(got, want))
    dw.close()


def test_cloth_mixed_1000_steps_within_1e6_of_f64(device, oracle):
    b, j, p = scenarios.cloth_world(5, 10, tol=1e-10, precision=PRECISION_MIXED)
    dw = _lib.DeviceWorld(device, b, j, p)
    dw.step(1000)
    q = p.copy()
    q["precision"] = PRECISION_F64
    ow = oracle.OracleWorld(b, j, q)
    ow.step(1000)
    err = pose_rel(dw.bodies(), ow.bodies())
    assert int(dw.stats()["fatal"]) == 0
    assert err <= 1e-6, err
    dw.close()


def worst_coordinate(bodies):
    pos = motors_np.apply_point_n(bodies["pose"], np.zeros((len(bodies), 3)))
    return float(np.abs(pos).max()) if np.isfinite(pos).all() else float("inf")


def test_cloth_survives_frame_time_spikes(device):
    """cloth_grid_stability.rs:130-153: 60 Hz frames with every 17th at 0.1 s; the curtain stays a
    hanging rag (every coordinate below 5 m) at the reference's own Newton tolerance."""
    b, j, p = scenarios.cloth_world(2, 4)
    dw = _lib.DeviceWorld(device, b, j, p)
    for frame in range(100):
        dw.set_epoch(0.1 if frame % 17 == 16 else 1.0 / 60.0)
        dw.step(1)
        assert worst_coordinate(dw.bodies()) < 5.0, frame
    dw.close()


@pytest.mark.parametrize("dt", [1.0, 10.0])
def test_cloth_survives_absurdly_large_steps(device, dt):
    """cloth_grid_stability.rs:155-193: one huge step, then a second of 60 Hz frames; the curtain
    stays finite and within 100 m after both."""
    b, j, p = scenarios.cloth_world(2, 4)
    dw = _lib.DeviceWorld(device, b, j, p)
    dw.set_epoch(dt)
    dw.step(1)
    after = worst_coordinate(dw.bodies())
    dw.set_epoch(1.0 / 60.0)
    dw.step(60)
    settled = worst_coordinate(dw.bodies())
    assert after < 100.0 and settled < 100.0, (after, settled)
    dw.close()


def test_cloth_and_trees_in_one_batch_step_as_alone(device):
    worlds = []
    for k, (c, r) in enumerate(((3, 6), (5, 10), (4, 8))):
        worlds.append(scenarios.cloth_world(c, r, tol=1e-10, precision=PRECISION_MIXED))
        tb, tj = scenarios.tree_world(60 + 40 * k, seed=500 + k)
        worlds.append((tb, tj, step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10,
                                           exact_jacobian=True)))
    batch = _lib.DeviceBatch(device, worlds)
    batch.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 32)  # trees on the wave, curtains on the island kernel
    batch.step(5)
    for k, (b, j, p) in enumerate(worlds):
        alone = _lib.DeviceWorld(device, b, j, p)
        alone.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 32)
        alone.step(5)
        got, want = batch.world_bodies(k), alone.bodies()
        assert np.array_equal(got["pose"], want["pose"]) and np.array_equal(got["momentum"], want["momentum"]), k
        alone.close()
    batch.close()
