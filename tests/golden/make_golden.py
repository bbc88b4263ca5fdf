"""Generates tests/golden/oracle_vectors.npz: seeded inputs and the f64 oracle's outputs for the
hot path's stages and for whole worlds, committed so that the parity tests have fixed targets.

Why these are oracle outputs and not the reference's: the reference (a Rust workspace whose build
needs a Vulkan device) cannot be built or run in this container or on the GPU box, and its own test
suite stores no golden vectors (its checks compute their expectations at test time). The oracle
itself is pinned against the reference's known-answer tests and properties (test_oracle_kat.py,
test_seam_oracle.py). These fixtures add two things: `test_golden.py` fails if the oracle's
arithmetic drifts from what was committed, and `test_gpu_golden.py` compares the CUDA path with
the committed numbers without running the oracle.

Every case stores its inputs as the library's records (bodies, joints, step parameters), so the
tests never regenerate inputs (numpy's transcendental functions may differ in the last bit across
CPUs); `scenarios` is only used here, once.

Run: python tests/golden/make_golden.py   (rewrites oracle_vectors.npz; needs oracle/_build)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))                   # tests/ (oracle_lib)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))  # repo root (exgame_b200)

import oracle_lib as orc  # noqa: E402
from exgame_b200 import scenarios  # noqa: E402
from exgame_b200.abi import (GRAVITY_OFF, GRAVITY_PLUMMER, GRAVITY_SIZE_CORE, JOINT_DTYPE, LIE_EULER,  # noqa: E402
                             NEWTON, step_params)

OUT = os.path.join(HERE, "oracle_vectors.npz")
FORMAT = 1

# whole-world cases: name -> (bodies, joints, params, steps); the oracle's exact solver. Each is the
# input of a live-oracle parity test of the CUDA path, so the GPU test's bounds are those tests' bounds.
WORLD_CASES = ("lie_gravity", "lie_chain", "newton_chain", "newton_tree_kinematic", "newton_islands_gravity",
               "curtain_exact", "newton_exact_pose_factor")


def joint_stage_inputs(seed=3, nb=40, nj=40):
    """Random poses and twists and joints of every law between random pairs: the joint-stage parity
    test's recipe and draws (its first 40 joints)."""
    rng = np.random.default_rng(seed)
    poses = np.array([orc.twist_exp(rng.normal(size=6)) for _ in range(nb)])
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
    return poses, vels, joints


def world_cases():
    none = np.zeros(0, dtype=JOINT_DTYPE)
    cases = {}
    cases["lie_gravity"] = (scenarios.gravity_world(200, 20.0, seed=4), none,
                            step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, softening=0.05, dt=1e-3),
                            100)
    b, j = scenarios.chain_world(12, seed=5)
    j["law"][::4] = 1  # the critically damped law too
    cases["lie_chain"] = (b, j, step_params(integrator=LIE_EULER, gravity_law=GRAVITY_OFF, dt=1e-3), 200)
    b, j = scenarios.chain_world(33, seed=53)
    cases["newton_chain"] = (b, j, step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10), 20)
    b, j = scenarios.tree_world(40, seed=31)
    b[5]["kinematic"] = 1
    b[5]["mass"] = 0.0
    cases["newton_tree_kinematic"] = (b, j, step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2, tol=1e-10),
                                      10)
    parts = [scenarios.chain_world(5, seed=40 + k, origin=(0, 30.0 * k, 0)) for k in range(6)]
    b, j = scenarios.concat_worlds(parts)
    cases["newton_islands_gravity"] = (b, j, step_params(integrator=NEWTON, gravity_law=GRAVITY_PLUMMER, softening=0.05,
                                                         G=1.0, dt=1e-2, tol=1e-10), 10)
    b, j, p = scenarios.cloth_world(3, 6, tol=1e-10)
    cases["curtain_exact"] = (b, j, p, 60)
    b, j = scenarios.tree_world(60, seed=61)
    cases["newton_exact_pose_factor"] = (b, j, step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=1e-2,
                                                           tol=1e-10, exact_jacobian=True), 10)
    assert tuple(cases) == WORLD_CASES
    return cases


def generate():
    out = {"format": np.array(FORMAT)}
    # gravity stage: forces on every body of a 300-body world under both laws
    g = scenarios.gravity_world(300, 20.0, seed=300)
    out["gravity_bodies"] = g
    out["gravity_plummer"] = orc.gravity_forces(g, GRAVITY_PLUMMER, 1.0, 0.05)
    gs = g.copy()
    gs["size"] *= 3.0  # the size core active for some pairs
    out["gravity_size_core_bodies"] = gs
    out["gravity_size_core"] = orc.gravity_forces(gs, GRAVITY_SIZE_CORE, 1.0, 0.05)
    # joint stage: values (12 per joint) and Jacobian blocks (12 x 25 per joint) at dt 0.016, warp 1.3
    poses, vels, joints = joint_stage_inputs()
    out["joint_poses"], out["joint_twists"], out["joint_records"] = poses, vels, joints
    plain, jac = [], []
    for jr in joints:
        args = (int(jr["law"]), jr["params"], poses[jr["a"]], poses[jr["b"]], vels[jr["a"]], vels[jr["b"]], 0.016, 1.3)
        plain.append(orc.plain_eval(*args))
        jac.append(orc.jacobian_eval(*args))
    out["joint_plain"], out["joint_jacobian"] = np.array(plain), np.array(jac)
    # whole worlds
    for name, (b, j, p, steps) in world_cases().items():
        ow = orc.OracleWorld(b, j, p)
        ow.step(steps)
        out[f"{name}.bodies"] = b
        out[f"{name}.joints"] = j
        out[f"{name}.params"] = np.ascontiguousarray(p).reshape(())
        out[f"{name}.steps"] = np.array(steps)
        out[f"{name}.final"] = ow.bodies()
        out[f"{name}.energy"] = np.array(ow.energy())
    return out


if __name__ == "__main__":
    data = generate()
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes, {len(data)} arrays)", file=sys.stderr)
