"""The wave schedule of the device Newton step (large islands: every phase a grid-wide kernel over
all such islands, per-island control between the phases).

Pins: forced onto small worlds, the wave schedule matches the oracle exactly as the island kernel
does (chains, trees with kinematic bodies, many islands with gravity, sub-division of a stiff
step, the exact mid-point factor); its states agree with the island kernel's to rounding; a world
stepped by the wave inside a batch or a pool is bit-identical to the same world stepped alone.
"""
import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import GRAVITY_OFF, GRAVITY_PLUMMER, JOINT_DTYPE, LIE_EULER, NEWTON, PRECISION_MIXED, step_params
from test_gpu_parity import state_error

pytestmark = pytest.mark.gpu

W = _lib.DeviceWorld


def wave_world(device, bodies, joints, params, min_bodies=1):
    w = _lib.DeviceWorld(device, bodies, joints, params)
    w.set_option(W.OPT_WAVE_MIN_BODIES, min_bodies)
    return w


def run_wave(oracle, device, bodies, joints, params, steps):
    ow = oracle.OracleWorld(bodies, joints, params)
    ow.step(steps)
    dw = wave_world(device, bodies, joints, params)
    dw.step(steps)
    assert dw.get_option(W.OPT_LAST_WAVE_ROUNDS) > 0  # the wave schedule ran
    return ow, dw


@pytest.mark.parametrize("n", [2, 8, 33])
def test_wave_chain_matches_oracle(device, oracle, n):
    bodies, joints = scenarios.chain_world(n, seed=20 + n)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10)
    ow, dw = run_wave(oracle, device, bodies, joints, params, 20)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)
    st = dw.stats()
    assert st["fatal"] == 0 and st["last_spans"] >= 1 and st["last_newton_iterations"] >= 1


def test_wave_tree_and_kinematic_matches_oracle(device, oracle):
    bodies, joints = scenarios.tree_world(40, seed=31)
    bodies[5]["kinematic"] = 1
    bodies[5]["mass"] = 0.0
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10)
    ow, dw = run_wave(oracle, device, bodies, joints, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)


def test_wave_many_islands_and_gravity(device, oracle):
    parts = [scenarios.chain_world(5, seed=40 + k, origin=(0, 30.0 * k, 0)) for k in range(6)]
    bodies, joints = scenarios.concat_worlds(parts)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_PLUMMER, softening=0.05, G=1.0, dt=1e-2, tol=1e-10)
    ow, dw = run_wave(oracle, device, bodies, joints, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)


def test_wave_stiff_step_subdivides_like_oracle(device, oracle):
    from test_oracle_kat import body, spring
    bs = np.array([body((1, 0, 0), (0, 50, 0)), body((-1, 0, 0), (0, -50, 0))])
    js = np.array([spring(0, 1, 2.0, 5e4, 5.0)])
    params = step_params(integrator=NEWTON, dt=0.02)
    ow, dw = run_wave(oracle, device, bs, js, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-7 and me < 1e-6, (pe, me)
    assert dw.stats()["last_spans"] >= 1


def test_wave_exact_pose_factor_matches_oracle(device, oracle):
    bodies, joints = scenarios.tree_world(60, seed=61)
    params = step_params(integrator=NEWTON, dt=1e-2, tol=1e-10, exact_jacobian=True)
    ow, dw = run_wave(oracle, device, bodies, joints, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)


@pytest.mark.parametrize("precision,ns", [(0, False), (PRECISION_MIXED, False), (PRECISION_MIXED, True)])
def test_wave_agrees_with_island_kernel(device, precision, ns):
    bodies, joints = scenarios.tree_world(700, seed=71)
    params = step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10, exact_jacobian=True,
                         ns_pivot=ns)
    a = _lib.DeviceWorld(device, bodies, joints, params)
    a.set_option(W.OPT_WAVE_MIN_BODIES, 1 << 20)  # island kernel
    a.step(5)
    b = wave_world(device, bodies, joints, params)
    b.step(5)
    # the same per-item arithmetic in both schedules: the states agree bit for bit
    x, y = a.bodies(), b.bodies()
    assert np.array_equal(x["pose"], y["pose"]) and np.array_equal(x["momentum"], y["momentum"])
    sa, sb = a.stats(), b.stats()
    assert sa["last_newton_iterations"] == sb["last_newton_iterations"]
    assert sa["last_spans"] == sb["last_spans"]


@pytest.mark.parametrize("precision,ns", [(0, False), (PRECISION_MIXED, False), (PRECISION_MIXED, True)])
def test_wave_batch_is_bitwise_identical_to_worlds_alone(device, precision, ns):
    worlds = []
    for k, n in enumerate([3, 50, 300, 900]):
        b, j = scenarios.tree_world(n, seed=80 + k)
        worlds.append((b, j, step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10, ns_pivot=ns)))
    b, j = scenarios.chain_world(40, seed=90)
    worlds.append((b, j, step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10, ns_pivot=ns)))
    worlds.append((scenarios.gravity_world(500, 30.0, seed=91), np.zeros(0, dtype=JOINT_DTYPE),
                   step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=precision,
                               softening=0.05, dt=1e-3)))
    batch = _lib.DeviceBatch(device, worlds)
    batch.set_option(W.OPT_WAVE_MIN_BODIES, 40)  # the three larger trees and the chain take the wave
    batch.step(4)
    for k, (b, j, p) in enumerate(worlds):
        alone = wave_world(device, b, j, p, min_bodies=40)
        alone.step(4)
        got = batch.world_bodies(k)
        want = alone.bodies()
        assert np.array_equal(got["pose"], want["pose"]) and np.array_equal(got["momentum"], want["momentum"]), k
        alone.close()


def test_wave_in_a_pool_with_churn(device):
    trees = [scenarios.tree_world(n, seed=100 + n) for n in (20, 600, 150, 900)]
    p = step_params(integrator=NEWTON, dt=1e-2, tol=1e-10)
    pool = _lib.DevicePool(device, max_bodies=4096, max_joints=8192, max_worlds=4)
    pool.set_option(W.OPT_WAVE_MIN_BODIES, 100)
    s0 = pool.admit(*trees[0], p)
    s1 = pool.admit(*trees[1], p)
    pool.step(2)
    pool.release(s0)
    s2 = pool.admit(*trees[2], p)
    pool.set_steps(s1, 1)  # s1 holds after one more step
    pool.step(3)
    for slot, (b, j), steps in ((s1, trees[1], 3), (s2, trees[2], 3)):
        alone = wave_world(device, b, j, p, min_bodies=100)
        alone.step(steps)
        got, want = pool.world_bodies(slot), alone.bodies()
        assert np.array_equal(got["pose"], want["pose"]) and np.array_equal(got["momentum"], want["momentum"])
        alone.close()
    pool.close()


def test_host_driven_rounds_equal_the_conditional_graph(device):
    """The profiler-friendly form (rounds replayed from the host) steps bit-identically to the
    conditional graph, and reports its round count."""
    worlds = []
    for k, n in enumerate((40, 400, 1200)):
        b, j = scenarios.tree_world(n, seed=120 + k)
        worlds.append((b, j, step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10,
                                         exact_jacobian=True)))
    out = []
    for host in (0, 1):
        batch = _lib.DeviceBatch(device, worlds)
        batch.set_option(W.OPT_WAVE_MIN_BODIES, 1)
        batch.set_option(W.OPT_WAVE_HOST_ROUNDS, host)
        batch.step(3)
        assert batch.get_option(W.OPT_LAST_WAVE_ROUNDS) > 0
        out.append(batch.bodies())
        batch.close()
    assert np.array_equal(out[0]["pose"], out[1]["pose"]) and np.array_equal(out[0]["momentum"], out[1]["momentum"])


@pytest.mark.parametrize("ns", [False, True])
def test_wide_and_narrow_elimination_levels_agree_with_island_kernel(device, ns):
    """A batch whose widest elimination levels hold more than 8192 nodes, so the wave eliminates
    them one thread per node and the narrow levels one warp per node: every world ends bit for bit
    as the island kernel leaves it (with Gauss-Jordan and with Newton-Schulz pivot inverses)."""
    worlds = []
    for k in range(64):
        b, j = scenarios.tree_world(2048, seed=400 + k)
        worlds.append((b, j, step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10,
                                         exact_jacobian=True, ns_pivot=ns)))
    a = _lib.DeviceBatch(device, worlds)
    a.set_option(W.OPT_WAVE_MIN_BODIES, 1 << 20)  # island kernel
    a.step(3)
    b = _lib.DeviceBatch(device, worlds)
    b.set_option(W.OPT_WAVE_MIN_BODIES, 1)
    b.step(3)
    # the batch exercises both elimination kernels: a level wider than 8192 nodes and one narrower
    assert b.get_option(W.OPT_WAVE_LEVEL_MAX_WIDTH) > 8192
    assert 0 < b.get_option(W.OPT_WAVE_LEVEL_MIN_WIDTH) <= 8192
    x, y = a.bodies(), b.bodies()
    assert np.array_equal(x["pose"], y["pose"]) and np.array_equal(x["momentum"], y["momentum"])
    a.close()
    b.close()
