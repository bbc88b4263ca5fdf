"""Parity at the configurations' own sizes and lengths: the CUDA path against the f64 oracle on
the same seeded inputs, each quantity's error stated.

  config 1  the 256-body chain, FP64 with the reference's Newton matrix, all 500 steps, on both
            Newton schedules;
  config 2  the 65,536-body gravity world and the 16 chains, mixed precision, a few full-size steps;
  config 3  the largest gravity world (8192 bodies) for 1000 steps, mixed precision; the largest
            tree for 20 steps and a 200-body tree for 1000 steps, mixed precision.

Error measures (per world): pose, per body, max |d pose| / max(1, max |pose|) over the motor's
eight components, then the worst body; momentum, max |d p| over the world's largest |p|; energy,
|E(device state) - E(oracle state)| / |E(oracle state)| with one energy function (the oracle's)
applied to both. The accuracy bound of the mixed path is 1e-6 relative pose error after 1000 steps. Set
EXG_ERROR_LOG to a file path to have each test append its measured errors there as JSON lines.
"""
import json
import os

import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import JOINT_DTYPE, PRECISION_F64, PRECISION_MIXED

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc(oracle):
    oracle.lib().orc_set_threads(os.cpu_count() or 1)
    yield oracle
    oracle.lib().orc_set_threads(1)


def errors(got, want, joints, params, oracle):
    gp, wp = got["pose"], want["pose"]
    pose = float((np.abs(gp - wp).max(axis=1) / np.maximum(1.0, np.abs(wp).max(axis=1))).max())
    pm = np.abs(want["momentum"]).max()
    mom = float(np.abs(got["momentum"] - want["momentum"]).max() / max(pm, 1e-300))
    e_want = oracle.OracleWorld(want, joints, params).energy()
    e_got = oracle.OracleWorld(got, joints, params).energy()
    energy = abs(e_got - e_want) / max(abs(e_want), 1e-300)
    return {"pose_rel": pose, "momentum_rel": mom, "energy_rel": float(energy)}


def log(name, **kv):
    path = os.environ.get("EXG_ERROR_LOG")
    line = dict(test=name, **kv)
    print(json.dumps(line))
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(line) + "\n")


@pytest.mark.parametrize("schedule", ["island", "wave"])
def test_config1_chain_all_500_steps_f64(device, orc, schedule):
    bodies, joints, params, steps = scenarios.config1()
    assert steps == 500 and len(bodies) == 256
    ow = orc.OracleWorld(bodies, joints, params)
    ow.step(steps)
    dw = _lib.DeviceWorld(device, bodies, joints, params)
    if schedule == "wave":
        dw.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 1)
        dw.set_option(_lib.DeviceWorld.OPT_WAVE_MAX_LEVELS, 1 << 20)
    dw.step(steps)
    err = errors(dw.bodies(), ow.bodies(), joints, params, orc)
    log("config1_chain_500_steps_f64_" + schedule, steps=steps, **err)
    assert int(dw.stats()["fatal"]) == 0
    assert err["pose_rel"] <= 1e-9 and err["momentum_rel"] <= 1e-8 and err["energy_rel"] <= 1e-9, err
    dw.close()


def test_config2_full_size_mixed_each_quantity(device, orc):
    """Each quantity's error of the mixed path against the f64 oracle on config 2 at full size.
    Gravity agrees to rounding. The chains' first step sits at the margin of the 1e-10 Newton
    tolerance: the Newton matrix (the reference's, without the rotated mass block's derivative)
    converges linearly there, so whether a chain's first span converges or is sub-divided depends
    on rounding; the oracle itself sub-divides one chain of the sixteen, and the device path (FP64 as
    well as mixed) sub-divides a different set. Two valid integrations of that step then differ by
    the mid-point rule's own error: about 1e-5 of the largest momentum, 1e-9 in pose (the mixed
    path's accuracy bound is 1e-6 relative pose error)."""
    (gb, gj, gp), (cb, cj, cp), _ = scenarios.config2_parts(precision=PRECISION_MIXED, exact_jacobian=True)
    assert len(gb) == 65536 and len(cb) == 16 * 256
    steps = 3
    batch = _lib.DeviceBatch(device, [(gb, gj, gp), (cb, cj, cp)])
    batch.step(steps)
    out = {}
    for k, (b, j, p) in enumerate(((gb, gj, gp), (cb, cj, cp))):
        q = p.copy()
        q["precision"] = PRECISION_F64
        ow = orc.OracleWorld(b, j, q)
        ow.step(steps)
        out["gravity" if k == 0 else "chains"] = errors(batch.world_bodies(k), ow.bodies(), j, q, orc)
    log("config2_full_size_mixed", steps=steps, **out)
    assert out["gravity"]["pose_rel"] <= 1e-12 and out["chains"]["pose_rel"] <= 1e-7, out
    assert out["gravity"]["momentum_rel"] <= 1e-8 and out["chains"]["momentum_rel"] <= 1e-4, out
    assert out["gravity"]["energy_rel"] <= 1e-12 and out["chains"]["energy_rel"] <= 1e-6, out
    batch.close()


def config3_pick(kind, rank_from_top=0):
    sizes = scenarios.config3_sizes(4096, seed=3)
    idx = np.arange(len(sizes))
    sel = idx[idx % 2 == (0 if kind == "gravity" else 1)]
    order = sel[np.argsort(-sizes[sel], kind="stable")]
    return int(order[rank_from_top]), sizes


def config3_world(k):
    (b, j, p), = scenarios.config3_worlds(4096, seed=3, precision=PRECISION_MIXED, exact_jacobian=True, only=[k])
    return b, j, p


def run_pair(device, orc, b, j, p, steps):
    dw = _lib.DeviceWorld(device, b, j, p)
    dw.step(steps)
    q = p.copy()
    q["precision"] = PRECISION_F64
    ow = orc.OracleWorld(b, j, q)
    ow.step(steps)
    err = errors(dw.bodies(), ow.bodies(), j, q, orc)
    fatal = int(dw.stats()["fatal"])
    dw.close()
    return err, fatal


def test_config3_largest_gravity_world_1000_steps_within_1e6(device, orc):
    k, sizes = config3_pick("gravity")
    b, j, p = config3_world(k)
    assert len(b) == sizes[k] and len(b) > 7000
    err, fatal = run_pair(device, orc, b, j, p, 1000)
    log("config3_largest_gravity_1000_steps_mixed", world=k, bodies=len(b), steps=1000, **err)
    assert fatal == 0
    assert err["pose_rel"] <= 1e-6, err


def test_config3_largest_tree_mixed(device, orc):
    k, sizes = config3_pick("tree")
    b, j, p = config3_world(k)
    assert len(b) > 7000
    err, fatal = run_pair(device, orc, b, j, p, 20)
    log("config3_largest_tree_20_steps_mixed", world=k, bodies=len(b), steps=20, **err)
    assert fatal == 0
    assert err["pose_rel"] <= 1e-9 and err["momentum_rel"] <= 1e-7, err


def test_config3_tree_1000_steps_mixed(device, orc):
    sizes = scenarios.config3_sizes(4096, seed=3)
    trees = [i for i in range(1, len(sizes), 2) if 190 <= sizes[i] <= 230]
    k = trees[0]
    b, j, p = config3_world(k)
    err, fatal = run_pair(device, orc, b, j, p, 1000)
    log("config3_tree_1000_steps_mixed", world=k, bodies=len(b), steps=1000, **err)
    assert fatal == 0
    assert err["pose_rel"] <= 1e-6, err
