"""The committed golden vectors (tests/golden/oracle_vectors.npz, made by tests/golden/make_golden.py)
against the oracle as built now: stage outputs and whole-world final states must be reproduced bit
for bit, whatever the oracle's thread count (its parallel loops own disjoint rows, islands and
worlds, and no reduction crosses threads). A failure means the oracle's arithmetic changed; the
fixtures are then regenerated on purpose, never loosened."""
import os

import numpy as np
import pytest

from exgame_b200 import scenarios
from exgame_b200.abi import GRAVITY_PLUMMER, GRAVITY_SIZE_CORE

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "oracle_vectors.npz")
WORLD_CASES = ("lie_gravity", "lie_chain", "newton_chain", "newton_tree_kinematic", "newton_islands_gravity",
               "curtain_exact", "newton_exact_pose_factor")


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        data = {k: d[k] for k in d.files}
    assert int(data["format"]) == 1
    return data


def test_fixture_lists_every_case(golden):
    for name in WORLD_CASES:
        for part in ("bodies", "joints", "params", "steps", "final", "energy"):
            assert f"{name}.{part}" in golden, (name, part)
    assert golden["joint_jacobian"].shape == (len(golden["joint_records"]), 12, 25)


def test_gravity_stage_reproduced(oracle, golden):
    got = oracle.gravity_forces(golden["gravity_bodies"], GRAVITY_PLUMMER, 1.0, 0.05)
    assert np.array_equal(got, golden["gravity_plummer"])
    got = oracle.gravity_forces(golden["gravity_size_core_bodies"], GRAVITY_SIZE_CORE, 1.0, 0.05)
    assert np.array_equal(got, golden["gravity_size_core"])


def test_joint_stage_reproduced(oracle, golden):
    poses, vels = golden["joint_poses"], golden["joint_twists"]
    for k, jr in enumerate(golden["joint_records"]):
        args = (int(jr["law"]), jr["params"], poses[jr["a"]], poses[jr["b"]], vels[jr["a"]], vels[jr["b"]], 0.016, 1.3)
        assert np.array_equal(oracle.plain_eval(*args), golden["joint_plain"][k]), k
        assert np.array_equal(oracle.jacobian_eval(*args), golden["joint_jacobian"][k]), k


@pytest.mark.parametrize("name", WORLD_CASES)
def test_world_reproduced(oracle, golden, name):
    ow = oracle.OracleWorld(golden[f"{name}.bodies"], golden[f"{name}.joints"], golden[f"{name}.params"])
    ow.step(int(golden[f"{name}.steps"]))
    got, want = ow.bodies(), golden[f"{name}.final"]
    assert np.array_equal(got["pose"], want["pose"]) and np.array_equal(got["momentum"], want["momentum"])
    assert ow.energy() == float(golden[f"{name}.energy"])


def test_worlds_reproduced_stepped_together(oracle, golden):
    """The oracle's world-parallel stepping (the CPU baseline's path) gives the same bits."""
    worlds = [oracle.OracleWorld(golden[f"{n}.bodies"], golden[f"{n}.joints"], golden[f"{n}.params"])
              for n in WORLD_CASES if int(golden[f"{n}.steps"]) == 10]
    assert len(worlds) == 3
    oracle.worlds_step(worlds, 10)
    for w, n in zip(worlds, [n for n in WORLD_CASES if int(golden[f"{n}.steps"]) == 10]):
        assert np.array_equal(w.bodies()["pose"], golden[f"{n}.final"]["pose"]), n


def test_fixture_inputs_come_from_the_committed_generators(golden):
    """The stored inputs are what the scenario generators make for the stored seeds (to rounding:
    numpy's transcendental functions may differ in the last bit across CPUs)."""
    g = scenarios.gravity_world(300, 20.0, seed=300)
    assert np.allclose(g["pose"], golden["gravity_bodies"]["pose"], rtol=0, atol=1e-13)
    assert np.array_equal(g["mass"], golden["gravity_bodies"]["mass"])
    b, j, _ = scenarios.cloth_world(3, 6, tol=1e-10)
    assert np.array_equal(j, golden["curtain_exact.joints"])
    assert np.allclose(b["pose"], golden["curtain_exact.bodies"]["pose"], rtol=0, atol=1e-13)
