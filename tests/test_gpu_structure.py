"""Bit-exact solver structure: the integer maps the device kernels index by, read back from the
device (exg_world_island_structure), against the oracle's restatement of the reference's island
partition, dynamic order (crates/newton/src/integrator/implicit/cache.rs:566-573) and gather
incidence (bake_incidence, crates/newton/src/accelerator/mod.rs:289-331): connection order, end a
before end b. Compared integer for integer with np.array_equal on chains, random trees, worlds of
several islands, kinematic bodies, batches and after joint replacement."""
import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import GRAVITY_OFF, JOINT_DTYPE, NEWTON, PRECISION_F64, PRECISION_MIXED, step_params

pytestmark = pytest.mark.gpu

EXACT_KINDS = ("bodies", "joints", "joint_ends", "order", "incidence_ptr", "incidence")


def implicit(precision=PRECISION_F64):
    return step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=1e-2, tol=1e-10)


def check_parents(dev_world, world, island, ends, order):
    """The elimination parents form a spanning forest of the island's dynamic joint graph: each
    parent edge is a joint between two dynamic bodies and every dynamic component has one root."""
    par = dev_world.island_structure(island, "parent", world)
    m = int((order >= 0).sum())
    assert len(par) == m
    adj = set()
    for law, a, b in ends:
        ia, ib = order[a], order[b]
        if ia >= 0 and ib >= 0:
            adj.add((ia, ib))
            adj.add((ib, ia))
    cyclic = len(adj) // 2 > m - 1
    for i, p in enumerate(par):
        # a tree island's parents are joint edges; a cyclic island's are its factor's (fill included)
        assert p == -1 or cyclic or (i, p) in adj
    # no cycles: following parents from any node reaches a root within m hops
    for i in range(m):
        x, hops = i, 0
        while par[x] != -1:
            x, hops = par[x], hops + 1
            assert hops <= m
    # one root per dynamic component
    comp = list(range(m))

    def find(x):
        while comp[x] != x:
            comp[x] = comp[comp[x]]
            x = comp[x]
        return x
    for a, b in adj:
        ra, rb = find(a), find(b)
        if ra != rb:
            comp[max(ra, rb)] = min(ra, rb)
    roots = {find(i) for i in range(m) if par[i] == -1}
    assert len(roots) == len({find(i) for i in range(m)}) == int((par == -1).sum())


def compare(dev_world, oracle, bodies, joints, params, world=0):
    ow = oracle.OracleWorld(bodies, joints, params)
    n_isl = dev_world.island_count(world)
    assert n_isl == ow.island_count()
    for k in range(n_isl):
        for kind in EXACT_KINDS:
            got, want = dev_world.island_structure(k, kind, world), ow.island_structure(k, kind)
            assert got.dtype.kind == "i" and np.array_equal(got, want.astype(got.dtype)), (world, k, kind)
        check_parents(dev_world, world, k, ow.island_structure(k, "joint_ends"), ow.island_structure(k, "order"))
    return n_isl


def with_kinematic(bodies, which):
    b = bodies.copy()
    b["kinematic"][which] = 1
    return b


def test_chain_and_tree_structure_is_the_oracles(device, oracle):
    for bodies, joints in (scenarios.chain_world(64, seed=11), scenarios.tree_world(300, seed=12),
                           scenarios.tree_world(2000, seed=13)):
        w = _lib.DeviceWorld(device, bodies, joints, implicit())
        assert compare(w, oracle, bodies, joints, implicit()) == 1
        w.close()


def test_several_islands_and_lone_bodies(device, oracle):
    parts = [scenarios.chain_world(12, seed=21), scenarios.tree_world(40, seed=22), scenarios.chain_world(1, seed=23),
             scenarios.tree_world(25, seed=24)]
    bodies, joints = scenarios.concat_worlds(parts)
    # interleave the joints of different islands: islands list their joints ascending
    perm = np.random.default_rng(5).permutation(len(joints))
    joints = joints[perm]
    w = _lib.DeviceWorld(device, bodies, joints, implicit())
    assert compare(w, oracle, bodies, joints, implicit()) == 4
    w.close()


def test_kinematic_bodies_leave_the_dynamic_order(device, oracle):
    bodies, joints = scenarios.tree_world(400, seed=31)
    bodies = with_kinematic(bodies, [0, 7, 19, 200, 399])
    w = _lib.DeviceWorld(device, bodies, joints, implicit(PRECISION_MIXED))
    w.step(1)
    compare(w, oracle, bodies, joints, implicit(PRECISION_MIXED))
    w.close()


def test_batch_worlds_and_joint_replacement(device, oracle):
    worlds = []
    for k, n in enumerate((20, 150, 700)):
        b, j = scenarios.tree_world(n, seed=40 + k)
        worlds.append((b, j, implicit(PRECISION_MIXED)))
    batch = _lib.DeviceBatch(device, worlds)
    batch.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 64)  # both schedules in one batch
    batch.step(1)
    for k, (b, j, p) in enumerate(worlds):
        compare(batch, oracle, b, j, p, world=k)
    # detach one edge's joints of world 2 (the tree splits in two) and connect world 1 across
    b2, j2, p2 = worlds[2]
    cut = j2[(j2["a"] != j2["a"][30]) | (j2["b"] != j2["b"][30])]
    batch.set_joints(cut, world=2)
    b1, j1, p1 = worlds[1]
    extra = np.zeros(10, dtype=JOINT_DTYPE)  # more joints than the batch has room for
    extra[:] = j1[0]
    extra["a"], extra["b"] = 3, 140
    j1b = np.concatenate([j1[:5], extra, j1[5:]])
    with pytest.raises(_lib.ExgError):  # beyond the batch's joint capacity: refused, nothing changes
        batch.set_joints(j1b, world=1)
    batch.step(1)
    assert compare(batch, oracle, b2, cut, p2, world=2) == 2
    compare(batch, oracle, b1, j1, p1, world=1)
    # the same count with an edge moved so that it closes a cycle: accepted (block-LU island)
    j1c = j1.copy()
    j1c[-1]["a"], j1c[-1]["b"] = 3, 140
    batch.set_joints(j1c, world=1)
    batch.step(1)
    compare(batch, oracle, b1, j1c, p1, world=1)
    batch.close()


def test_cloth_islands_structure(device, oracle):
    """A curtain's dynamic bodies form cycles: the island keeps the oracle's gather maps and order
    (the block-LU solve changes only the elimination structure)."""
    b, j, p = scenarios.cloth_world(5, 10, tol=1e-10)
    w = _lib.DeviceWorld(device, b, j, p)
    w.step(1)
    assert compare(w, oracle, b, j, p) == 1
    w.close()
