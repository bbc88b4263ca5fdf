"""The launch-shape autotuner: every tuned value leaves results bit-identical, and the tuner picks
one of its candidates for each knob."""
import numpy as np
import pytest

from exgame_b200 import _lib, autotune, scenarios
from exgame_b200.abi import GRAVITY_PLUMMER, JOINT_DTYPE, LIE_EULER, NEWTON, PRECISION_MIXED, step_params

pytestmark = pytest.mark.gpu
D = _lib.Device


def mixed_batch():
    worlds = [(scenarios.gravity_world(3000, 50.0, seed=1), np.zeros(0, dtype=JOINT_DTYPE),
               step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=PRECISION_MIXED,
                           softening=0.05, dt=1e-3))]
    for k, n in enumerate((20, 300, 900)):
        b, j = scenarios.tree_world(n, seed=30 + k)
        worlds.append((b, j, step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10,
                                         exact_jacobian=True)))
    return worlds


def run(device, worlds, g, w, t, n=8192):
    device.set_tuning(D.TUNE_GRAVITY_CTAS_PER_SM, g)
    device.set_tuning(D.TUNE_WAVE_BLOCKS_PER_SM, w)
    device.set_tuning(D.TUNE_WAVE_MIN_BODIES, t)
    device.set_tuning(D.TUNE_WAVE_NARROW_LEVEL, n)
    batch = _lib.DeviceBatch(device, worlds)
    batch.step(3)
    out = batch.bodies()
    batch.close()
    return out


def test_tuning_never_changes_results(device):
    worlds = mixed_batch()
    defaults = [device.get_tuning(k) for k in (1, 2, 3, 4)]
    try:
        ref = run(device, worlds, 32, 8, 32)
        for g, w, t, n in ((8, 4, 1, 1), (21, 16, 256, 1 << 30), (1, 1, 1 << 20, 64), (32, 8, 1, 1 << 30)):
            got = run(device, worlds, g, w, t, n)
            assert np.array_equal(got["pose"], ref["pose"]) and np.array_equal(got["momentum"], ref["momentum"])
    finally:
        for k, v in zip((1, 2, 3, 4), defaults):
            device.set_tuning(k, v)


def test_autotune_picks_candidates(device):
    defaults = [device.get_tuning(k) for k in (1, 2, 3, 4)]
    try:
        r = autotune.autotune(device, gravity_bodies=8192, trees=8, tree_bodies=600, steps=2)
        assert r["wave_narrow_level"] in autotune.NARROW_LEVELS
        assert r["gravity_ctas_per_sm"] in autotune.GRAVITY_CTAS
        assert r["wave_blocks_per_sm"] in autotune.WAVE_BLOCKS
        assert r["wave_min_bodies"] in autotune.WAVE_THRESHOLDS
        assert device.get_tuning(D.TUNE_GRAVITY_CTAS_PER_SM) == r["gravity_ctas_per_sm"]
        with pytest.raises(_lib.ExgError):
            device.set_tuning(D.TUNE_GRAVITY_CTAS_PER_SM, 0)
    finally:
        for k, v in zip((1, 2, 3, 4), defaults):
            device.set_tuning(k, v)


def test_autotune_on_a_workload_keeps_its_results(device):
    """Timed on the caller's own batch: the tuned batch, after the tuner's steps and as many more,
    holds the same bits as an untuned copy stepped as often."""
    defaults = [device.get_tuning(k) for k in (1, 2, 3, 4)]
    p = step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10, exact_jacobian=True)
    worlds = [(*scenarios.tree_world(n, seed=70 + k), p) for k, n in enumerate((30, 200, 900))]
    g = scenarios.gravity_world(2048, 100.0, seed=77)
    worlds.append((g, np.zeros(0, dtype=JOINT_DTYPE),
                   step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=PRECISION_MIXED,
                               softening=0.05, dt=1e-3)))
    try:
        tuned = _lib.DeviceBatch(device, worlds)
        r = autotune.autotune(device, workload=tuned, steps=1)
        assert r["timed_on"] == "workload" and r["wave_min_bodies"] in autotune.WAVE_THRESHOLDS
        n_steps = 2 * (len(autotune.GRAVITY_CTAS) + len(autotune.WAVE_BLOCKS) + len(autotune.WAVE_THRESHOLDS) +
                       len(autotune.NARROW_LEVELS))
        tuned.step(3)
        plain = _lib.DeviceBatch(device, worlds)
        plain.step(n_steps + 3)
        for k in range(len(worlds)):
            a, b = tuned.world_bodies(k), plain.world_bodies(k)
            assert np.array_equal(a["pose"], b["pose"]) and np.array_equal(a["momentum"], b["momentum"]), k
        tuned.close()
        plain.close()
    finally:
        for k, v in zip((1, 2, 3, 4), defaults):
            device.set_tuning(k, v)


def test_tuning_cache_hit_sets_the_tuned_values(device, tmp_path):
    """A second process-like call on a batch of the same shape reads the cache instead of timing:
    same choices, set on the device and the handle, and the handle's state untouched."""
    defaults = [device.get_tuning(k) for k in (1, 2, 3, 4)]
    p = step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10, exact_jacobian=True)
    worlds = [(*scenarios.tree_world(n, seed=90 + k), p) for k, n in enumerate((40, 300))]
    path = str(tmp_path / "tuning.json")
    try:
        first = _lib.DeviceBatch(device, worlds)
        r1 = autotune.autotune(device, workload=first, steps=1, cache=path)
        first.close()
        assert r1["timed_on"] == "workload"
        for k, v in zip((1, 2, 3, 4), defaults):
            device.set_tuning(k, v)
        second = _lib.DeviceBatch(device, worlds)
        before = second.bodies()
        launches = device.kernel_launches()
        r2 = autotune.autotune(device, workload=second, steps=1, cache=path)
        assert r2["timed_on"] == "cache" and device.kernel_launches() == launches
        for name, key, _ in autotune.KNOBS:
            assert r2[name] == r1[name] and device.get_tuning(key) == r1[name]
        after = second.bodies()
        assert np.array_equal(before["pose"], after["pose"])
        second.close()
    finally:
        for k, v in zip((1, 2, 3, 4), defaults):
            device.set_tuning(k, v)
