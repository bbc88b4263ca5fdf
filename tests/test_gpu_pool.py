"""Pools and the request loop: worlds admitted and released while others step, and served requests.

Pins: a world stepped inside a pool — admitted late, beside worlds that come and go, with its
ranges reused from released worlds — ends bit-identical to the same world stepped alone (the
reference's driver-vs-solo property, crates/newton/tests/ar0103_epoch_driver.rs:115-158); a
world's step budget stops it after exactly that many steps; a served request's result is the same
alone and in the mix.
"""
import threading

import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import (GRAVITY_PLUMMER, GRAVITY_SIZE_CORE, JOINT_DTYPE, LIE_EULER, NEWTON, PRECISION_F64,
                             PRECISION_MIXED, SYMPLECTIC_EULER, step_params)

pytestmark = pytest.mark.gpu


def world_set(precision=PRECISION_F64):
    out = []
    for k, n in enumerate([5, 300, 40, 1500]):
        p = step_params(integrator=LIE_EULER if k % 2 == 0 else SYMPLECTIC_EULER,
                        gravity_law=GRAVITY_PLUMMER if k % 2 == 0 else GRAVITY_SIZE_CORE,
                        precision=precision, softening=0.05, dt=1e-3)
        out.append((scenarios.gravity_world(n, 30.0, seed=500 + k), np.zeros(0, dtype=JOINT_DTYPE), p))
    for k, n in enumerate([3, 60, 257]):
        b, j = scenarios.tree_world(n, seed=600 + k)
        out.append((b, j, step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10)))
    b, j = scenarios.chain_world(33, seed=700)
    out.append((b, j, step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10)))
    return out


def alone(device, world, steps):
    b, j, p = world
    w = _lib.DeviceWorld(device, b, j, p)
    w.step(steps)
    out = w.bodies()
    w.close()
    return out


def same(a, b):
    return np.array_equal(a["pose"], b["pose"]) and np.array_equal(a["momentum"], b["momentum"])


@pytest.mark.parametrize("precision", [PRECISION_F64, PRECISION_MIXED])
def test_pool_with_churn_is_bitwise_identical_to_worlds_alone(device, precision):
    worlds = world_set(precision)
    pool = _lib.DevicePool(device, max_bodies=4096, max_joints=4096, max_worlds=8, precision=precision)
    slots = {}
    for k in (0, 1, 4, 5, 7):
        slots[k] = pool.admit(*worlds[k])
    pool.step(3)
    pool.release(slots.pop(1))  # frees a 300-body range in the middle
    pool.release(slots.pop(5))
    for k in (2, 6, 3):          # admitted into reused ranges, and one past them
        slots[k] = pool.admit(*worlds[k])
    pool.step(4)
    ran = {0: 7, 4: 7, 7: 7, 2: 4, 6: 4, 3: 4}
    for k, steps in ran.items():
        assert same(pool.world_bodies(slots[k]), alone(device, worlds[k], steps)), k
    pool.close()


def test_pool_step_budget_holds_a_world_exactly(device):
    worlds = world_set()
    pool = _lib.DevicePool(device, max_bodies=4096, max_joints=4096, max_worlds=8)
    s0 = pool.admit(*worlds[1])
    s1 = pool.admit(*worlds[5])
    s2 = pool.admit(*worlds[7])
    pool.set_steps(s0, 2)
    pool.set_steps(s1, 5)
    pool.step(6)  # s2 is unbounded
    left = pool.steps_left(8)
    assert left[s0] == 0 and left[s1] == 0 and left[s2] == -1
    assert same(pool.world_bodies(s0), alone(device, worlds[1], 2))
    assert same(pool.world_bodies(s1), alone(device, worlds[5], 5))
    assert same(pool.world_bodies(s2), alone(device, worlds[7], 6))
    pool.close()


def test_pool_capacity_errors_leave_it_usable(device):
    worlds = world_set()
    pool = _lib.DevicePool(device, max_bodies=400, max_joints=400, max_worlds=2)
    s = pool.admit(*worlds[1])   # 300 bodies
    s2 = pool.admit(*worlds[5])  # 60 bodies: both world slots now used
    with pytest.raises(_lib.ExgError) as e:
        pool.admit(*worlds[2])
    assert e.value.name == "EXG_ERR_OUT_OF_MEMORY"  # no world slot
    pool.release(s2)
    with pytest.raises(_lib.ExgError) as e:
        pool.admit(*worlds[6])  # 257 bodies: no body range long enough
    assert e.value.name == "EXG_ERR_OUT_OF_MEMORY"
    s2 = pool.admit(*worlds[5])
    with pytest.raises(_lib.ExgError) as e:
        pool.release(7)
    assert e.value.name == "EXG_ERR_INVALID_ARGUMENT"
    with pytest.raises(_lib.ExgError):
        pool.admit(*world_set(PRECISION_MIXED)[0])  # precision differs from the pool's
    u = pool.usage()
    assert u["worlds_used"] == 2 and u["worlds_capacity"] == 2
    pool.step(2)
    assert same(pool.world_bodies(s), alone(device, worlds[1], 2))
    pool.close()


@pytest.mark.parametrize("pools", [1, 2])
@pytest.mark.parametrize("precision", [PRECISION_F64, PRECISION_MIXED])
def test_served_results_are_the_same_alone_and_in_the_mix(device, precision, pools):
    """Requests of uneven size and step count submitted from two threads while others run; each
    result equals the same world stepped alone for its step count, bit for bit, with one pool and
    with two pools whose ticks overlap on the GPU."""
    worlds = world_set(precision)
    steps = [7, 31, 3, 50, 12, 1, 26, 40]
    srv = _lib.Server(device, max_bodies=8192, max_joints=8192, max_worlds=16, precision=precision,
                      steps_per_tick=8, pools=pools)
    ids = [None] * len(worlds)

    def producer(ks):
        for k in ks:
            ids[k] = srv.submit(*worlds[k], steps[k])

    t = threading.Thread(target=producer, args=([1, 3, 5, 7],))
    t.start()
    producer([0, 2, 4, 6])
    t.join()
    for k in range(len(worlds)):
        res = srv.wait(ids[k], timeout_ms=120000)
        assert res is not None, k
        out, info = res
        assert info["status"] == 0 and info["steps"] == steps[k]
        assert same(out, alone(device, worlds[k], steps[k])), k
    st = srv.stats()
    assert st["completed"] == len(worlds) and st["failed"] == 0 and st["queued"] == 0 and st["running"] == 0
    assert st["body_steps"] == sum(len(w[0]) * s for w, s in zip(worlds, steps))
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0
    srv.close()


def test_server_admits_against_the_budget(device):
    """A budget that holds one world at a time still serves every request, one after another."""
    worlds = world_set()
    fp = max(_lib.world_footprint(len(b), len(j), p) for b, j, p in worlds)
    srv = _lib.Server(device, hbm_budget_bytes=fp, max_bodies=8192, max_joints=8192, max_worlds=16,
                      steps_per_tick=4)
    ids = [srv.submit(*w, 5) for w in worlds]
    for k, rid in enumerate(ids):
        out, info = srv.wait(rid, timeout_ms=120000)
        assert same(out, alone(device, worlds[k], 5)), k
    st = srv.stats()
    assert st["peak_resident_bytes"] <= fp and st["completed"] == len(worlds)
    assert not srv.sizes  # nothing left pending
    with pytest.raises(_lib.ExgError) as e:  # larger than the whole budget: refused at submission
        srv.submit(*scenarios.tree_world(4000, seed=9), step_params(integrator=NEWTON), 3)
    assert e.value.name == "EXG_ERR_OUT_OF_MEMORY"
    srv.close()


def test_server_poll_and_zero_step_requests(device):
    worlds = world_set()
    srv = _lib.Server(device, max_bodies=4096, max_joints=4096, max_worlds=4, steps_per_tick=2)
    r0 = srv.submit(*worlds[0], 0)
    out, info = srv.wait(r0, timeout_ms=60000)
    assert same(out, worlds[0][0])
    r1 = srv.submit(*worlds[6], 3)
    res = None
    for _ in range(20000):
        res = srv.poll(r1)
        if res is not None:
            break
    if res is None:
        res = srv.wait(r1, timeout_ms=120000)
    assert same(res[0], alone(device, worlds[6], 3))
    with pytest.raises(_lib.ExgError):
        srv.poll(r1)  # collected already: unknown id
    srv.close()


def test_whole_handle_records_follow_slot_order_through_page_locked_buffers(device):
    """exg_world_get/set_bodies on a pool with a released slot in the middle: the records are the
    used slots in slot order, and a page-locked buffer round-trips them exactly."""
    worlds = world_set()
    pool = _lib.DevicePool(device, max_bodies=4096, max_joints=4096, max_worlds=8)
    s = [pool.admit(*worlds[k]) for k in (1, 2, 5, 6)]
    pool.release(s[1])
    pool.step(2)
    buf = _lib.host_bodies(pool.n)
    pool.bodies(out=buf)
    want = np.concatenate([pool.world_bodies(k) for k in sorted(pool.counts)])
    assert same(buf, want)
    buf["momentum"] *= 0.5
    pool.set_bodies(buf)
    back = pool.bodies()
    assert same(back, buf)
    k = sorted(pool.counts)[1]
    assert same(pool.world_bodies(k), buf[pool.counts[sorted(pool.counts)[0]]:][:pool.counts[k]])
    pool.close()


def test_state_accessors_move_pose_and_momentum_in_record_order(device):
    """exg_world_get/set_state on a pool with a released slot in the middle: 14 doubles per body
    (pose then momentum) in the records' order; setting states changes nothing else, and stepping
    from them equals stepping from the same records set whole."""
    worlds = world_set()
    pool = _lib.DevicePool(device, max_bodies=4096, max_joints=4096, max_worlds=8)
    s = [pool.admit(*worlds[k]) for k in (1, 2, 5, 6)]
    pool.release(s[1])
    pool.step(2)
    rec = pool.bodies()
    st = _lib.host_state(pool.n)
    pool.state(out=st)
    assert np.array_equal(st[:, :8], rec["pose"]) and np.array_equal(st[:, 8:], rec["momentum"])
    st[:, 8:] *= 0.5
    pool.set_state(st)
    back = pool.bodies()
    assert np.array_equal(back["momentum"], st[:, 8:]) and np.array_equal(back["pose"], st[:, :8])
    for f in ("mass", "inertia", "size", "kinematic", "diagonal"):
        assert np.array_equal(back[f], rec[f]), f
    pool.step(3)
    via_state = pool.bodies()
    rec["momentum"] *= 0.5
    pool.set_bodies(rec)
    pool.step(3)
    assert same(pool.bodies(), via_state)
    with pytest.raises(ValueError):
        pool.set_state(st[:-1])
    pool.close()


def test_server_fails_a_non_finite_world_and_serves_the_rest(device):
    """A request whose world is not finite (a NaN momentum) fails with EXG_ERR_FATAL (the
    reference's EvalError::Fatal of a guarded site), while the requests beside it complete and
    equal their worlds stepped alone."""
    worlds = world_set()
    bad_b, bad_j, bad_p = worlds[6]
    bad_b = bad_b.copy()
    bad_b["momentum"][3, 0] = np.nan
    srv = _lib.Server(device, max_bodies=8192, max_joints=8192, max_worlds=8, steps_per_tick=4)
    good = [srv.submit(*worlds[k], 6) for k in (1, 5, 7)]
    bad = srv.submit(bad_b, bad_j, bad_p, 6)
    for k, rid in zip((1, 5, 7), good):
        out, info = srv.wait(rid, timeout_ms=120000)
        assert same(out, alone(device, worlds[k], 6)), k
    with pytest.raises(_lib.ExgError) as e:
        srv.wait(bad, timeout_ms=120000)
    assert e.value.name == "EXG_ERR_FATAL"
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 3
    # the loop is still serving
    out, _ = srv.wait(srv.submit(*worlds[0], 2), timeout_ms=60000)
    assert same(out, alone(device, worlds[0], 2))
    srv.close()
