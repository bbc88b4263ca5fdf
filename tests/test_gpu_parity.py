"""Parity of the CUDA path (through the C ABI) with the oracle on the same seeded inputs.

Tolerances: the FP64 path agrees with the f64 oracle to rounding (rtol 1e-12 per stage, 1e-9 on
states after many steps); the mixed path is bounded by its FP32 stages (stated per test). Integer
structure (topology, incidence, ordering) is bit-exact by construction: the kernels consume the
records as given.
"""
import ctypes

import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import (GRAVITY_OFF, GRAVITY_PLUMMER, GRAVITY_SIZE_CORE, JOINT_DTYPE, LIE_EULER, NEWTON,
                             PRECISION_F64, PRECISION_MIXED, PRECISION_MIXED_FAST, SYMPLECTIC_EULER, EXPLICIT_EULER,
                             step_params)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dev_tensor(a):
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).cuda()
    torch.cuda.synchronize()
    return t


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def positions(bodies):
    return np.array([_lib.motor_apply_point(b["pose"], np.zeros(3)) for b in bodies])


def pos_mass(bodies):
    p = positions(bodies)
    pm = np.zeros((len(bodies), 4))
    pm[:, :3] = p
    pm[:, 3] = np.where(bodies["kinematic"] != 0, 0.0, bodies["mass"])
    return pm


@pytest.mark.parametrize("law", [GRAVITY_SIZE_CORE, GRAVITY_PLUMMER])
@pytest.mark.parametrize("n", [1, 7, 300, 5000])
def test_gravity_stage_fp64_matches_oracle(device, oracle, law, n):
    bodies = scenarios.gravity_world(n, 20.0, seed=n)
    if n > 1 and law == GRAVITY_SIZE_CORE:
        bodies["size"] *= 3.0  # make the size core active for some pairs
    pm = pos_mass(bodies)
    d_pm, d_size = dev_tensor(pm), dev_tensor(np.ascontiguousarray(bodies["size"]))
    d_f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().exg_gravity_forces(device.handle, vp(d_pm), vp(d_size), n, law, 1.0, 0.05, PRECISION_F64,
                                             vp(d_f)))
    got = d_f.cpu().numpy().reshape(n, 3)
    want = oracle.gravity_forces(bodies, law, 1.0, 0.05)
    scale = np.abs(want).max() + 1e-300
    assert np.abs(got - want).max() <= 1e-12 * scale


@pytest.mark.parametrize("precision", [PRECISION_MIXED, PRECISION_MIXED_FAST])
@pytest.mark.parametrize("law", [GRAVITY_SIZE_CORE, GRAVITY_PLUMMER])
def test_gravity_stage_mixed_error_bound(device, oracle, law, precision):
    """FP32 pair terms (on double-single separations in MIXED, tile-relative FP32 positions in
    MIXED_FAST) and FP64 tile accumulation. Bounds: median per-body relative force error below
    1e-6, and every body's error below 5e-5 of the root mean square force (a body whose pulls
    nearly cancel has a small net force, so its own relative error is not the right yardstick)."""
    n = 4096
    bodies = scenarios.gravity_world(n, 1000.0, seed=9)
    pm = pos_mass(bodies)
    d_pm, d_size = dev_tensor(pm), dev_tensor(np.ascontiguousarray(bodies["size"]))
    d_f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().exg_gravity_forces(device.handle, vp(d_pm), vp(d_size), n, law, 1.0, 0.05, precision,
                                             vp(d_f)))
    got = d_f.cpu().numpy().reshape(n, 3)
    want = oracle.gravity_forces(bodies, law, 1.0, 0.05)
    err = np.linalg.norm(got - want, axis=1)
    mag = np.linalg.norm(want, axis=1)
    assert np.median(err / mag) < 1e-6, np.median(err / mag)
    rms = np.sqrt(np.mean(mag ** 2))
    assert (err / rms).max() < 5e-5, (err / rms).max()


@pytest.mark.parametrize("jacobian", [0, 1])
def test_joint_stage_matches_oracle(device, oracle, jacobian):
    rng = np.random.default_rng(3)
    nb, nj = 40, 120
    poses = np.array([oracle.twist_exp(rng.normal(size=6)) for _ in range(nb)])
    vels = rng.normal(size=(nb, 6))
    joints = np.zeros(nj, dtype=JOINT_DTYPE)
    for k in range(nj):
        law = k % 4
        a, b = rng.choice(nb, 2, replace=False)
        joints[k]["law"], joints[k]["a"], joints[k]["b"] = law, a, b
        if law <= 1:
            joints[k]["params"][:10] = np.r_[rng.normal(size=6) * 0.3, 1.3, 7.0, 2.0, 1e-6]
        elif law == 2:
            joints[k]["params"][:2] = [2.0, 1e-3]
        else:
            joints[k]["params"][0] = 1.5
    width = 300 if jacobian else 12
    d_j, d_p, d_v = dev_tensor(joints), dev_tensor(poses), dev_tensor(vels)
    d_out = torch.zeros(nj * width, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().exg_eval_joints(device.handle, vp(d_j), nj, vp(d_p), vp(d_v), 0.016, 1.3, jacobian, vp(d_out)))
    got = d_out.cpu().numpy().reshape(nj, width)
    for k in range(nj):
        j = joints[k]
        args = (int(j["law"]), j["params"], poses[j["a"]], poses[j["b"]], vels[j["a"]], vels[j["b"]], 0.016, 1.3)
        want = oracle.jacobian_eval(*args).reshape(-1) if jacobian else oracle.plain_eval(*args)
        assert np.allclose(got[k], want, rtol=1e-12, atol=1e-12), k


def run_both(oracle, device, bodies, joints, params, steps, solver=0):
    ow = oracle.OracleWorld(bodies, joints, params, solver=solver)
    ow.step(steps)
    dw = _lib.DeviceWorld(device, bodies, joints, params)
    dw.step(steps)
    return ow, dw


def state_error(a, b):
    pa, pb = positions(a), positions(b)
    scale = max(1.0, np.abs(pa).max())
    pos_err = np.abs(pa - pb).max() / scale
    mom_scale = max(1e-12, np.abs(a["momentum"]).max())
    mom_err = np.abs(a["momentum"] - b["momentum"]).max() / mom_scale
    return pos_err, mom_err


@pytest.mark.parametrize("scheme", [LIE_EULER, SYMPLECTIC_EULER, EXPLICIT_EULER])
@pytest.mark.parametrize("law", [GRAVITY_PLUMMER, GRAVITY_SIZE_CORE])
def test_explicit_gravity_world_matches_oracle(device, oracle, scheme, law):
    bodies = scenarios.gravity_world(200, 20.0, seed=4)
    params = step_params(integrator=scheme, gravity_law=law, softening=0.05, dt=1e-3)
    ow, dw = run_both(oracle, device, bodies, np.zeros(0, dtype=JOINT_DTYPE), params, 100)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-11 and me < 1e-10, (pe, me)


def test_explicit_jointed_world_matches_oracle(device, oracle):
    bodies, joints = scenarios.chain_world(12, seed=5)
    joints["law"][::4] = 1  # include the critically damped law
    params = step_params(integrator=LIE_EULER, gravity_law=GRAVITY_OFF, dt=1e-3)
    ow, dw = run_both(oracle, device, bodies, joints, params, 200)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-11 and me < 1e-9, (pe, me)


def test_config0_full_size_matches_oracle(device, oracle):
    """1024 bodies, Plummer 0.05, LieEuler, dt 1e-3, 1000 steps: final positions, velocities and
    total energy against the f64 oracle."""
    bodies, joints, params, steps = scenarios.config0()
    ow, dw = run_both(oracle, device, bodies, joints, params, steps)
    a, b = ow.bodies(), dw.bodies()
    pe, me = state_error(a, b)
    assert pe < 1e-9 and me < 1e-8, (pe, me)
    assert abs(ow.energy() - dw.energy()) <= 1e-9 * abs(ow.energy())
    # linear momentum is conserved by the pairwise law up to rounding
    p0 = bodies["momentum"][:, :3].sum(0)
    p1 = np.array([_lib.screw_transport(x["momentum"], x["pose"], 1)[:3] for x in b]).sum(0)
    assert np.abs(p1 - p0).max() < 1e-9 * np.abs(bodies["momentum"]).sum()


@pytest.mark.parametrize("n", [2, 8, 33])
def test_newton_chain_matches_oracle(device, oracle, n):
    bodies, joints = scenarios.chain_world(n, seed=20 + n)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10)
    ow, dw = run_both(oracle, device, bodies, joints, params, 20)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)
    st = dw.stats()
    assert st["fatal"] == 0 and st["last_spans"] >= 1


def test_newton_tree_and_kinematic_matches_oracle(device, oracle):
    bodies, joints = scenarios.tree_world(40, seed=31)
    bodies[5]["kinematic"] = 1
    bodies[5]["mass"] = 0.0
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10)
    ow, dw = run_both(oracle, device, bodies, joints, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)


def test_newton_many_islands_and_gravity(device, oracle):
    parts = [scenarios.chain_world(5, seed=40 + k, origin=(0, 30.0 * k, 0)) for k in range(6)]
    bodies, joints = scenarios.concat_worlds(parts)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_PLUMMER, softening=0.05, G=1.0, dt=1e-2, tol=1e-10)
    ow, dw = run_both(oracle, device, bodies, joints, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)


def test_newton_stiff_step_subdivides_like_oracle(device, oracle):
    """A stiff transverse pair at a coarse step (newton.rs:946-1027 geometry): the device reaches the
    oracle's state, sub-division included."""
    from test_oracle_kat import body, spring
    bs = np.array([body((1, 0, 0), (0, 50, 0)), body((-1, 0, 0), (0, -50, 0))])
    js = np.array([spring(0, 1, 2.0, 5e4, 5.0)])
    params = step_params(integrator=NEWTON, dt=0.02)
    ow, dw = run_both(oracle, device, bs, js, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-7 and me < 1e-6, (pe, me)


def test_config1_chain_first_steps_match_oracle(device, oracle):
    """The full 256-body chain (config 1): the first 5 steps against the oracle."""
    bodies, joints, params, _ = scenarios.config1()
    ow, dw = run_both(oracle, device, bodies, joints, params, 5)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)


def test_device_counts_kernel_launches(device):
    bodies = scenarios.gravity_world(64, 10.0, seed=1)
    dw = _lib.DeviceWorld(device, bodies, np.zeros(0, dtype=JOINT_DTYPE),
                          step_params(gravity_law=GRAVITY_PLUMMER, softening=0.05, dt=1e-3))
    before = device.kernel_launches()  # after the upload of the records (one scatter kernel)
    dw.step(3)
    assert device.kernel_launches() - before == 9  # pre, gravity, integrate per step


def test_newton_exact_pose_factor_matches_oracle(device, oracle):
    bodies, joints = scenarios.tree_world(60, seed=61)
    params = step_params(integrator=NEWTON, dt=1e-2, tol=1e-10, exact_jacobian=True)
    ow, dw = run_both(oracle, device, bodies, joints, params, 10)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)
    # and the same step as the reference's Newton matrix, within the tolerance
    ref = oracle.OracleWorld(bodies, joints, step_params(integrator=NEWTON, dt=1e-2, tol=1e-10))
    ref.step(10)
    pe, me = state_error(ref.bodies(), dw.bodies())
    assert pe < 1e-8 and me < 1e-6, (pe, me)


def test_newton_phase_cycles_reported(device):
    bodies, joints = scenarios.chain_world(30, seed=62)
    dw = _lib.DeviceWorld(device, bodies, joints, step_params(integrator=NEWTON, dt=1e-2, tol=1e-10))
    dw.step(2)
    ph = dw.phase_cycles()
    assert ph["joints+jacobian"] > 0 and ph["solve"] > 0 and ph["line search"] > 0


@pytest.mark.parametrize("scheme", [LIE_EULER, NEWTON])
def test_uniform_field_matches_oracle(device, oracle, scheme):
    """UniformField (field.rs:17-47) beside gravity: a jointed tree with a kinematic body in a field
    of weight plus a crosswind, explicit and implicit, both Newton schedules."""
    bodies, joints = scenarios.tree_world(30, seed=81)
    bodies[4]["kinematic"] = 1
    bodies[4]["mass"] = 0.0
    params = step_params(integrator=scheme, gravity_law=GRAVITY_PLUMMER, softening=0.05, dt=1e-2 if scheme == NEWTON else 1e-3,
                         tol=1e-10, field=(0.0, 1.5, -9.81))
    steps = 10 if scheme == NEWTON else 100
    ow = oracle.OracleWorld(bodies, joints, params)
    ow.step(steps)
    for min_bodies in ((1 << 20, 1) if scheme == NEWTON else (1 << 20,)):
        dw = _lib.DeviceWorld(device, bodies, joints, params)
        dw.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, min_bodies)
        dw.step(steps)
        pe, me = state_error(ow.bodies(), dw.bodies())
        assert pe < 1e-9 and me < 1e-7, (min_bodies, pe, me)
        dw.close()


def test_set_bodies_kinematic_change_rebuilds_islands(device, oracle):
    """Records set between steps may turn a body kinematic (or back): the implicit world's islands
    are rebuilt from the new flags, on both Newton schedules, and the steps that follow match an
    oracle world made from the same records; the batch accessor does the same for one world."""
    bodies, joints = scenarios.tree_world(40, seed=83)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10)
    for min_bodies in (1 << 20, 1):
        dw = _lib.DeviceWorld(device, bodies, joints, params)
        dw.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, min_bodies)
        dw.step(3)
        for kin, mass in ((1, 0.0), (0, bodies[7]["mass"])):
            rec = dw.bodies()
            rec[7]["kinematic"], rec[7]["mass"] = kin, mass
            dw.set_bodies(rec)
            ow = oracle.OracleWorld(rec, joints, params)
            dw.step(4)
            ow.step(4)
            pe, me = state_error(ow.bodies(), dw.bodies())
            assert pe < 1e-9 and me < 1e-7, (min_bodies, kin, pe, me)
        dw.close()
    other, oj = scenarios.chain_world(6, seed=84)
    batch = _lib.DeviceBatch(device, [(bodies, joints, params), (other, oj, params)])
    batch.step(2)
    rec = batch.world_bodies(0)
    rec[3]["kinematic"], rec[3]["mass"] = 1, 0.0
    batch.set_world_bodies(0, rec)
    ow = oracle.OracleWorld(rec, joints, params)
    batch.step(3)
    ow.step(3)
    pe, me = state_error(ow.bodies(), batch.world_bodies(0))
    assert pe < 1e-9 and me < 1e-7, (pe, me)
    batch.close()


def _edge_mask(joints, a, b):
    return ((joints["a"] == a) & (joints["b"] == b)) | ((joints["a"] == b) & (joints["b"] == a))


@pytest.mark.parametrize("scheme", [NEWTON, LIE_EULER])
def test_set_joints_detach_and_connect_match_oracle(device, oracle, scheme):
    """Joints replaced between steps (exg_batch_set_joints): detaching a tree edge splits an
    island, connecting it again merges the two; each following span matches an oracle world made
    from the current records and the new joints, on both Newton schedules and explicitly."""
    bodies, joints = scenarios.tree_world(40, seed=86)
    params = step_params(integrator=scheme, gravity_law=GRAVITY_OFF, dt=1e-2 if scheme == NEWTON else 1e-3,
                         tol=1e-10)
    c = 17  # its parent is its one neighbour of lower index (the generator's parents precede)
    touch = (joints["a"] == c) | (joints["b"] == c)
    ends = np.where(joints["a"][touch] == c, joints["b"][touch], joints["a"][touch])
    cut = joints[~_edge_mask(joints, c, int(ends[ends < c][0]))]
    assert len(cut) == len(joints) - 3
    steps = 4 if scheme == NEWTON else 40
    for min_bodies in ((1 << 20, 1) if scheme == NEWTON else (1 << 20,)):
        dw = _lib.DeviceWorld(device, bodies, joints, params)
        dw.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, min_bodies)
        dw.step(steps)
        for new in (cut, joints):
            dw.set_joints(new)
            ow = oracle.OracleWorld(dw.bodies(), new, params)
            dw.step(steps)
            ow.step(steps)
            pe, me = state_error(ow.bodies(), dw.bodies())
            assert pe < 1e-9 and me < 1e-7, (min_bodies, len(new), pe, me)
        dw.close()


def test_set_joints_closing_a_cycle_and_a_refused_list(device, oracle):
    """A joint list that closes a cycle of dynamic bodies moves the island to the block-LU solve
    and the world then steps as the oracle does; a list beyond the handle's joint capacity is
    refused (EXG_ERR_OUT_OF_MEMORY) and the world steps on exactly as an untouched twin; in a
    batch, replacing one world's joints leaves the other world bit for bit as when stepped alone."""
    bodies, joints = scenarios.tree_world(24, seed=87)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10)
    loop = joints.copy()  # same count (a world handle's joint capacity is its count at creation)
    loop[-1]["a"], loop[-1]["b"] = 5, 9  # the dropped law leaves its edge joined by the other two
    a = _lib.DeviceWorld(device, bodies, joints, params)
    b = _lib.DeviceWorld(device, bodies, joints, params)
    a.step(2)
    b.step(2)
    a.set_joints(loop)
    ow = oracle.OracleWorld(a.bodies(), loop, params)
    a.step(3)
    ow.step(3)
    pe, me = state_error(ow.bodies(), a.bodies())
    assert pe < 1e-9 and me < 1e-7, (pe, me)
    with pytest.raises(_lib.ExgError) as e:
        b.set_joints(np.concatenate([joints, joints[:1]]))
    assert e.value.status == -21  # EXG_ERR_OUT_OF_MEMORY: beyond the handle's joint capacity
    twin = _lib.DeviceWorld(device, bodies, joints, params)
    twin.step(2)
    b.step(3)
    twin.step(3)
    assert np.array_equal(b.bodies()["pose"], twin.bodies()["pose"])
    a.close()
    b.close()
    twin.close()
    other, oj = scenarios.chain_world(8, seed=88)
    batch = _lib.DeviceBatch(device, [(other, oj, params), (bodies, joints, params)])
    alone = _lib.DeviceWorld(device, other, oj, params)
    batch.step(2)
    ow = oracle.OracleWorld(batch.world_bodies(1), joints[3:], params)
    batch.set_joints(joints[3:], world=1)
    batch.step(3)
    alone.step(5)
    ow.step(3)
    assert np.array_equal(batch.world_bodies(0)["pose"], alone.bodies()["pose"])
    pe, me = state_error(ow.bodies(), batch.world_bodies(1))
    assert pe < 1e-9 and me < 1e-7, (pe, me)
    batch.close()
    alone.close()


def test_set_bodies_refuses_massless_dynamic_record(device):
    """A dynamic record without positive mass refuses exg_world_set_bodies as a whole: nothing of
    the call is written, and the world steps on from its previous state."""
    bodies, joints = scenarios.tree_world(20, seed=85)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10)
    dw = _lib.DeviceWorld(device, bodies, joints, params)
    dw.step(2)
    before = dw.bodies()
    rec = before.copy()
    rec["pose"][:, 0] += 1.0
    rec[5]["mass"] = 0.0
    with pytest.raises(_lib.ExgError):
        dw.set_bodies(rec)
    after = dw.bodies()
    assert np.array_equal(before["pose"], after["pose"]) and np.array_equal(before["mass"], after["mass"])
    dw.step(1)
    dw.close()


def test_mixed_gravity_world_1000_steps_within_1e6_of_f64(device, oracle):
    """The mixed path's accuracy target: a config-0 cluster (1024 bodies in a ball of radius 100,
    Plummer 0.05, LieEuler, dt 1e-3) after 1000 steps against the f64 oracle — relative pose
    error at most 1e-6. The single-FP32 form (MIXED_FAST) is stated beside it: its close pairs
    carry the rounding of their distance to the tile reference, which the cluster amplifies."""
    bodies = scenarios.gravity_world(1024, 100.0, seed=7)
    kw = dict(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, softening=0.05, dt=1e-3)
    ow = oracle.OracleWorld(bodies, np.zeros(0, dtype=JOINT_DTYPE), step_params(**kw))
    ow.step(1000)
    want = ow.bodies()
    dw = _lib.DeviceWorld(device, bodies, np.zeros(0, dtype=JOINT_DTYPE), step_params(precision=PRECISION_MIXED, **kw))
    dw.step(1000)
    pe, me = state_error(want, dw.bodies())
    assert pe <= 1e-6, pe
    fw = _lib.DeviceWorld(device, bodies, np.zeros(0, dtype=JOINT_DTYPE),
                          step_params(precision=PRECISION_MIXED_FAST, **kw))
    fw.step(1000)
    pf, mf = state_error(want, fw.bodies())
    assert pf < 1e-4 and pf > pe, (pf, pe)


def rotated_inertia(bodies, seed):
    """Each body's diagonal box inertia turned into a full tensor R diag R^T (random R): the
    general Inertia::Rigid path (crates/newton/src/inertia.rs:145-156, 271-345)."""
    rng = np.random.default_rng(seed)
    b = bodies.copy()
    for k in range(len(b)):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        d = np.diag([b[k]["inertia"][0], b[k]["inertia"][4], b[k]["inertia"][8]])
        full = q @ d @ q.T
        b[k]["inertia"] = (0.5 * (full + full.T)).reshape(9)
        b[k]["diagonal"] = 0
    b["momentum"][:, 3:] = rng.normal(size=(len(b), 3)) * 0.3  # spin, so the tensor matters
    return b


@pytest.mark.parametrize("precision", [PRECISION_F64, PRECISION_MIXED])
def test_full_inertia_tensor_newton_both_schedules(device, oracle, precision):
    bodies, joints = scenarios.tree_world(60, seed=91)
    bodies = rotated_inertia(bodies, 92)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=1e-2, tol=1e-10)
    ow = oracle.OracleWorld(bodies, joints, params)
    ow.step(20)
    out = []
    for min_bodies in (1 << 20, 1):
        dw = _lib.DeviceWorld(device, bodies, joints, params)
        dw.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, min_bodies)
        dw.step(20)
        pe, me = state_error(ow.bodies(), dw.bodies())
        assert pe < 1e-9 and me < 1e-7, (min_bodies, pe, me)
        out.append(dw.bodies())
        dw.close()
    assert np.array_equal(out[0]["pose"], out[1]["pose"])


@pytest.mark.parametrize("scheme", [LIE_EULER, SYMPLECTIC_EULER, EXPLICIT_EULER])
def test_full_inertia_tensor_explicit(device, oracle, scheme):
    bodies, joints = scenarios.chain_world(24, seed=93)
    bodies = rotated_inertia(bodies, 94)
    params = step_params(integrator=scheme, gravity_law=GRAVITY_PLUMMER, softening=0.05, dt=1e-3)
    ow, dw = run_both(oracle, device, bodies, joints, params, 50)
    pe, me = state_error(ow.bodies(), dw.bodies())
    assert pe < 1e-10 and me < 1e-9, (pe, me)
    dw.close()
