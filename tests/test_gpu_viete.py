"""Traced joint laws (exgame_b200/user_laws.py, compiled to the device by viete) on the GPU: the
stage call against the built-in law it restates, whole worlds on both Newton schedules against the
built-in law and the oracle, and the new PointBushing law stepping a tree (bit for bit the same on
the island kernel and the wave, world momentum conserved with internal forces only)."""
import ctypes

import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import JOINT_DTYPE, NEWTON, PRECISION_F64, PRECISION_MIXED, step_params

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TRACED_SPRING, _ = 4, 10
BUSHING = 5


def dev_tensor(a):
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()
    torch.cuda.synchronize()
    return t


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("jacobian", [0, 1])
def test_traced_law_stage_equals_the_built_in_law(device, oracle, jacobian):
    assert _lib.law_lookup("TracedSpringDamper") == (TRACED_SPRING, 10)
    rng = np.random.default_rng(5)
    nb, nj = 30, 60
    poses = np.array([oracle.twist_exp(rng.normal(size=6)) for _ in range(nb)])
    vels = rng.normal(size=(nb, 6))
    joints = np.zeros(nj, dtype=JOINT_DTYPE)
    for k in range(nj):
        a, b = rng.choice(nb, 2, replace=False)
        joints[k]["law"], joints[k]["a"], joints[k]["b"] = 0, a, b
        joints[k]["params"][:10] = np.r_[rng.normal(size=6) * 0.3, 1.3, 7.0, 2.0, 1e-6]
    traced = joints.copy()
    traced["law"] = TRACED_SPRING
    width = 300 if jacobian else 12
    d_p, d_v = dev_tensor(poses), dev_tensor(vels)
    outs = []
    for js in (joints, traced):
        d_j = dev_tensor(js)
        d_out = torch.zeros(nj * width, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        _lib.check(_lib.lib().exg_eval_joints(device.handle, vp(d_j), nj, vp(d_p), vp(d_v), 0.016, 1.3, jacobian,
                                              vp(d_out)))
        outs.append(d_out.cpu().numpy().reshape(nj, width))
    scale = np.abs(outs[0]).max()
    assert np.abs(outs[1] - outs[0]).max() <= 1e-12 * scale


@pytest.mark.parametrize("wave", [False, True])
def test_world_with_traced_springs_steps_as_the_built_in_law(device, oracle, wave):
    bodies, joints = scenarios.tree_world(120, seed=61)
    params = step_params(integrator=NEWTON, precision=PRECISION_F64, dt=1e-2, tol=1e-10)
    traced = joints.copy()
    traced["law"][traced["law"] == 0] = TRACED_SPRING
    a = _lib.DeviceWorld(device, bodies, joints, params)
    b = _lib.DeviceWorld(device, bodies, traced, params)
    for w in (a, b):
        w.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 1 if wave else 1 << 20)
        w.step(40)
    x, y = a.bodies(), b.bodies()
    scale = max(1.0, np.abs(x["pose"]).max())
    assert np.abs(x["pose"] - y["pose"]).max() <= 1e-11 * scale
    ow = oracle.OracleWorld(bodies, joints, params)
    ow.step(40)
    assert np.abs(ow.bodies()["pose"] - y["pose"]).max() <= 1e-9 * scale
    a.close()
    b.close()


def world_momentum(bodies):
    """Sum over bodies of the world-frame momentum (coAd of the body-frame momentum)."""
    tot = np.zeros(6)
    for b in bodies:
        tot += _lib.screw_transport(b["momentum"], b["pose"], 1)
    return tot


@pytest.mark.parametrize("precision", [PRECISION_F64, PRECISION_MIXED])
def test_point_bushing_tree_conserves_momentum_on_both_schedules(device, precision):
    assert _lib.law_lookup("PointBushing") == (BUSHING, 8)
    bodies, joints = scenarios.tree_world(80, seed=62, laws=(0,))
    rng = np.random.default_rng(9)
    bodies["momentum"] = rng.normal(size=(len(bodies), 6)) * 0.5
    bush = np.zeros(len(joints), dtype=JOINT_DTYPE)
    bush["law"], bush["a"], bush["b"] = BUSHING, joints["a"], joints["b"]
    # anchors at the body centres: a zero-length spring between them, damped
    bush["params"][:, 6] = 200.0
    bush["params"][:, 7] = 2.0
    params = step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10, exact_jacobian=True)
    out = []
    for min_bodies in (1 << 20, 1):
        w = _lib.DeviceWorld(device, bodies, bush, params)
        w.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, min_bodies)
        w.step(30)
        assert int(w.stats()["fatal"]) == 0
        out.append(w.bodies())
        w.close()
    assert np.array_equal(out[0]["pose"], out[1]["pose"]) and np.array_equal(out[0]["momentum"], out[1]["momentum"])
    p0, p1 = world_momentum(bodies), world_momentum(out[0])
    assert np.abs(p1 - p0).max() <= 1e-8 * max(1.0, np.abs(p0).max()), (p0, p1)
