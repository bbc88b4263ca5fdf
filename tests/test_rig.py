"""The hitchcock camera rig as a consumer workload of the implicit path (CPU: the scenario and the
oracle). The rig (crates/hitchcock/src/camera.rs:259-520) is four bodies per camera, 17 critically
damped axial springs, three torsional and two transverse dampers, and a kinematic tracker that the
host moves to the target before every step (camera.rs:55-76)."""
import numpy as np

from exgame_b200 import motors_np, scenarios


def rig_target(t, n, jump_at=2.0):
    """Rig k's target: a circle of radius 5 about (1000 k, 0, 0) at 0.5 rad/s, moved 10 along x
    at jump_at (a retarget: the tracker teleports and the springs pull the rig after it)."""
    w = 0.5
    c = np.array([[1000.0 * k, 0.0, 0.0] for k in range(n)])
    off = np.array([5.0 * np.cos(w * t) - 5.0, 5.0 * np.sin(w * t), 0.0])
    vel = np.array([-5.0 * w * np.sin(w * t), 5.0 * w * np.cos(w * t), 0.0])
    jump = np.array([10.0, 0.0, 0.0]) if t >= jump_at else np.zeros(3)
    return c + off + jump, np.tile(vel, (n, 1))


def state_of(bodies):
    return np.concatenate([bodies["pose"], bodies["momentum"]], axis=1)


def test_rig_layout():
    b, j, p = scenarios.camera_rig_world(3, r_object=2.0, linear=1.0)
    assert len(b) == 12 and len(j) == 66
    assert list(b["kinematic"]) == [0, 0, 0, 1] * 3
    per = j[:22]
    assert list(per["law"]) == [1] * 17 + [3] * 3 + [2] * 2
    assert list(zip(per["a"][17:], per["b"][17:])) == [(0, 1), (1, 2), (1, 3), (1, 3), (2, 3)]
    rests = per["params"][:17, 6]
    s1 = 2.0 * np.sqrt(2.0)
    assert np.allclose(rests, [0, 0, s1, s1] + [s1] * 8 + [2.0] * 5)
    assert (j["a"][22:44] >= 4).all() and (j["b"][22:44] < 8).all()  # rig 1 joins only its own bodies


def test_rig_follows_its_target_on_the_oracle(oracle):
    n = 2
    b, j, p = scenarios.camera_rig_world(n, r_object=2.0, linear=1.0)
    ow = oracle.OracleWorld(b, j, p)
    dt = float(p["dt"])
    for s in range(400):
        cur = ow.bodies()
        st = scenarios.track_targets(state_of(cur), n, *rig_target(s * dt, n))
        nb = cur.copy()
        nb["pose"], nb["momentum"] = st[:, :8], st[:, 8:]
        ow.set_state(nb)
        ow.step(1)
    end = ow.bodies()
    eye = motors_np.apply_point_n(end["pose"][0::4], np.zeros((n, 3)))
    tc, _ = rig_target(399 * dt, n)
    d = np.linalg.norm(eye - tc, axis=1)
    assert (d < 10.0).all() and np.allclose(d[0], d[1:], rtol=1e-6), d  # the rigs are alike
    assert np.isfinite(end["momentum"]).all()
