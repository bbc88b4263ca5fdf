"""The CUDA path (through the C ABI) against the committed golden vectors
(tests/golden/oracle_vectors.npz): the f64 oracle's outputs for the gravity and joint stages and
for whole worlds, stored with their inputs, so this test runs no oracle code. The bounds are those
of the live-oracle parity tests on the same inputs: stages to 1e-12, explicit worlds to 1e-11 in
position, implicit worlds to 1e-9 in position and 1e-7 in momentum, the curtain (block LU) to
1e-10 per body."""
import ctypes
import os

import numpy as np
import pytest

from exgame_b200 import _lib
from exgame_b200.abi import GRAVITY_PLUMMER, GRAVITY_SIZE_CORE, PRECISION_F64

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_vectors.npz")
# case -> (position bound, momentum bound) relative to the largest magnitude
WORLD_BOUNDS = {"lie_gravity": (1e-11, 1e-10), "lie_chain": (1e-11, 1e-9), "newton_chain": (1e-9, 1e-7),
                "newton_tree_kinematic": (1e-9, 1e-7), "newton_islands_gravity": (1e-9, 1e-7),
                "newton_exact_pose_factor": (1e-9, 1e-7)}


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def dev_tensor(a):
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()
    torch.cuda.synchronize()
    return t


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def positions(bodies):
    return np.array([_lib.motor_apply_point(b["pose"], np.zeros(3)) for b in bodies])


def state_error(want, got):
    pa, pb = positions(want), positions(got)
    pos_err = np.abs(pa - pb).max() / max(1.0, np.abs(pa).max())
    mom_err = np.abs(want["momentum"] - got["momentum"]).max() / max(1e-12, np.abs(want["momentum"]).max())
    return pos_err, mom_err


@pytest.mark.parametrize("law,key", [(GRAVITY_PLUMMER, "gravity"), (GRAVITY_SIZE_CORE, "gravity_size_core")])
def test_gravity_stage_matches_golden(device, golden, law, key):
    bodies = golden["gravity_bodies" if key == "gravity" else "gravity_size_core_bodies"]
    want = golden["gravity_plummer" if key == "gravity" else "gravity_size_core"]
    n = len(bodies)
    pm = np.zeros((n, 4))
    pm[:, :3] = positions(bodies)
    pm[:, 3] = np.where(bodies["kinematic"] != 0, 0.0, bodies["mass"])
    d_pm, d_size = dev_tensor(pm), dev_tensor(np.ascontiguousarray(bodies["size"]))
    d_f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().exg_gravity_forces(device.handle, vp(d_pm), vp(d_size), n, law, 1.0, 0.05, PRECISION_F64,
                                             vp(d_f)))
    got = d_f.cpu().numpy().reshape(n, 3)
    assert np.abs(got - want).max() <= 1e-12 * (np.abs(want).max() + 1e-300)


@pytest.mark.parametrize("jacobian", [0, 1])
def test_joint_stage_matches_golden(device, golden, jacobian):
    joints, poses, vels = golden["joint_records"], golden["joint_poses"], golden["joint_twists"]
    nj = len(joints)
    width = 300 if jacobian else 12
    d_j, d_p, d_v = dev_tensor(joints), dev_tensor(poses), dev_tensor(vels)
    d_out = torch.zeros(nj * width, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().exg_eval_joints(device.handle, vp(d_j), nj, vp(d_p), vp(d_v), 0.016, 1.3, jacobian,
                                          vp(d_out)))
    got = d_out.cpu().numpy().reshape(nj, width)
    want = golden["joint_jacobian"].reshape(nj, 300) if jacobian else golden["joint_plain"]
    for k in range(nj):
        assert np.allclose(got[k], want[k], rtol=1e-12, atol=1e-12), k


@pytest.mark.parametrize("name", sorted(WORLD_BOUNDS))
def test_world_matches_golden(device, golden, name):
    dw = _lib.DeviceWorld(device, golden[f"{name}.bodies"], golden[f"{name}.joints"], golden[f"{name}.params"])
    dw.step(int(golden[f"{name}.steps"]))
    got, want = dw.bodies(), golden[f"{name}.final"]
    pe, me = state_error(want, got)
    bp, bm = WORLD_BOUNDS[name]
    assert pe < bp and me < bm, (pe, me)
    assert int(dw.stats()["fatal"]) == 0
    if name == "lie_gravity":
        e = float(golden[f"{name}.energy"])
        assert abs(dw.energy() - e) <= 1e-9 * abs(e)
    dw.close()


def test_curtain_matches_golden(device, golden):
    """The cyclic island (block LU on the device) against the oracle's exact dense solve."""
    name = "curtain_exact"
    dw = _lib.DeviceWorld(device, golden[f"{name}.bodies"], golden[f"{name}.joints"], golden[f"{name}.params"])
    dw.step(int(golden[f"{name}.steps"]))
    got, want = dw.bodies(), golden[f"{name}.final"]
    assert int(dw.stats()["fatal"]) == 0
    pose_rel = float((np.abs(got["pose"] - want["pose"]).max(axis=1) /
                      np.maximum(1.0, np.abs(want["pose"]).max(axis=1))).max())
    mom_rel = float(np.abs(got["momentum"] - want["momentum"]).max() / max(np.abs(want["momentum"]).max(), 1e-300))
    assert pose_rel <= 1e-10 and mom_rel <= 1e-8, (pose_rel, mom_rel)
    dw.close()
