"""Batches: many independent worlds of uneven size stepped together.

Pins: every world of a batch is bit-identical to the same world stepped alone (the reference's
driver-vs-solo property, crates/newton/tests/ar0103_epoch_driver.rs:115-158; mechanisms of different
sizes sharing one accelerator, crates/newton/tests/concurrent_mechanisms.rs:84-137; and its
batch-policy independence, crates/newton/tests/ar0104_batch_determinism.rs:140-153), and matches the
oracle.
"""
import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import (GRAVITY_OFF, GRAVITY_PLUMMER, GRAVITY_SIZE_CORE, JOINT_DTYPE, LIE_EULER, NEWTON,
                             PRECISION_F64, PRECISION_MIXED, step_params)

pytestmark = pytest.mark.gpu


def mixed_worlds(precision=PRECISION_F64):
    worlds = []
    for k, n in enumerate([3, 200, 17, 1100, 64]):
        p = step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER if k % 2 == 0 else GRAVITY_SIZE_CORE,
                        precision=precision, softening=0.05, dt=1e-3)
        worlds.append((scenarios.gravity_world(n, 30.0, seed=100 + k), np.zeros(0, dtype=JOINT_DTYPE), p))
    for k, n in enumerate([2, 9, 40, 150]):
        b, j = scenarios.tree_world(n, seed=200 + k)
        worlds.append((b, j, step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10)))
    b, j = scenarios.chain_world(20, seed=300)
    worlds.append((b, j, step_params(integrator=NEWTON, precision=precision, dt=1e-2, tol=1e-10)))
    return worlds


def test_batch_is_bitwise_identical_to_worlds_alone(device):
    worlds = mixed_worlds()
    batch = _lib.DeviceBatch(device, worlds)
    batch.step(5)
    for k, (b, j, p) in enumerate(worlds):
        alone = _lib.DeviceWorld(device, b, j, p)
        alone.step(5)
        a, m = alone.bodies(), batch.world_bodies(k)
        assert np.array_equal(a["pose"], m["pose"]), k
        assert np.array_equal(a["momentum"], m["momentum"]), k
        alone.close()


def test_batch_matches_oracle(device, oracle):
    worlds = mixed_worlds()
    batch = _lib.DeviceBatch(device, worlds)
    batch.step(5)
    from test_gpu_parity import state_error
    for k, (b, j, p) in enumerate(worlds):
        ow = oracle.OracleWorld(b, j, p)
        ow.step(5)
        pe, me = state_error(ow.bodies(), batch.world_bodies(k))
        assert pe < 1e-9 and me < 1e-7, (k, pe, me)


def test_batch_world_accessors_roundtrip(device):
    worlds = mixed_worlds()
    batch = _lib.DeviceBatch(device, worlds)
    b3 = batch.world_bodies(3)
    b3["momentum"] *= 0.5
    batch.set_world_bodies(3, b3)
    assert np.array_equal(batch.world_bodies(3)["momentum"], b3["momentum"])
    assert np.array_equal(batch.bodies()[batch.offsets[3]:batch.offsets[4]]["momentum"], b3["momentum"])
    st = batch.world_stats(7)
    assert st["fatal"] == 0


def test_batch_mixed_precision_error_vs_oracle(device, oracle):
    """Mixed form (FP32 forces, FP64 pose / residual / solve): relative pose error vs the f64
    oracle after 20 steps, stated per world kind."""
    worlds = mixed_worlds(PRECISION_MIXED)
    batch = _lib.DeviceBatch(device, worlds)
    batch.step(20)
    from test_gpu_parity import state_error
    for k, (b, j, p) in enumerate(worlds):
        pf = p.copy()
        pf["precision"] = PRECISION_F64
        ow = oracle.OracleWorld(b, j, pf)
        ow.step(20)
        pe, me = state_error(ow.bodies(), batch.world_bodies(k))
        assert pe < 1e-6, (k, pe, me)


def test_config3_sized_batch_runs(device):
    """A 256-world slice of config 3 (sizes log-uniform in [8, 8192]) steps without a fatal status."""
    worlds = scenarios.config3_worlds(256, seed=3, precision=PRECISION_MIXED)
    batch = _lib.DeviceBatch(device, worlds)
    batch.step(2)
    st = batch.stats()
    assert st["fatal"] == 0
    out = batch.bodies()
    assert np.all(np.isfinite(out["pose"])) and np.all(np.isfinite(out["momentum"]))


def test_handles_on_their_own_streams_step_side_by_side_bit_for_bit(device):
    """Two batch handles with EXG_OPT_OWN_STREAM, each driven by its own host thread (state in,
    a step, state out, every step), end bit for bit where the same handles stepped one after the
    other on the device's stream end; a third handle on the device stream steps meanwhile."""
    import threading
    worlds = mixed_worlds(PRECISION_MIXED)
    halves = (worlds[:5], worlds[5:])
    want = []
    for part in halves:
        b = _lib.DeviceBatch(device, part)
        for _ in range(6):
            st = b.state()
            b.set_state(st)
            b.step(1)
        want.append(b.bodies())
        b.close()
    handles = [_lib.DeviceBatch(device, part) for part in halves]
    shared = _lib.DeviceBatch(device, worlds[:3])
    for h in handles:
        h.set_option(_lib.DeviceWorld.OPT_OWN_STREAM, 1)
        assert h.get_option(_lib.DeviceWorld.OPT_OWN_STREAM) == 1
    assert handles[0].stream() != handles[1].stream() != shared.stream()
    errors = []

    def drive(h):
        try:
            st = _lib.host_state(h.n)
            for _ in range(6):
                h.state(out=st)
                h.set_state(st)
                h.step(1)
        except Exception as e:  # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=drive, args=(h,)) for h in handles]
    for t in threads:
        t.start()
    shared.step(4)
    for t in threads:
        t.join()
    assert not errors, errors
    for h, w in zip(handles, want):
        got = h.bodies()
        assert np.array_equal(got["pose"], w["pose"]) and np.array_equal(got["momentum"], w["momentum"])
        h.set_option(_lib.DeviceWorld.OPT_OWN_STREAM, 0)
        h.close()
    shared.close()
