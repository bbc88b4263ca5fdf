"""Seeded synthetic workloads (the reference ships no benchmark data; these stand in for the
configurations the measurements are quoted on).

Every generator draws from numpy's PCG64 (`numpy.random.default_rng(seed)`) and returns host
arrays in the C ABI's record layouts (BODY_DTYPE, JOINT_DTYPE) plus step parameters. Motors are
built with a numpy restatement of the motor algebra (motors_np), so generating a workload loads
no part of the CUDA library.

  gravity_world  N point masses: positions uniform in a ball, masses log-uniform in [1, 10],
                 circular-orbit speed about the centre of mass (mass strictly inside the radius
                 counted exactly) perpendicular to r about the z axis (a random axis when r is
                 parallel to z), plus N(0, 0.01) per component.
  chain_world    boxes with half-extents U[0.5, 2], density 1 (m = 8 hx hy hz,
                 I = m/3 (hy^2+hz^2, hx^2+hz^2, hx^2+hy^2)), CoM-to-CoM along x and touching;
                 each adjacent pair carries an axial SimpleSpringDamper (anchors at the CoMs,
                 rest = initial distance, k log-uniform in [1e2, 1e4], c = 0.1 sqrt(k),
                 softening 1e-6), a PerpendicularDamperWarped (c, 1e-6) and a
                 TorsionalDamperWarped (c); each motor is exp(xi) followed by the placement,
                 xi ~ N(0, 0.05) per twist component; bodies start at rest.
  tree_world     as chain_world, but body i > 0 hangs from a parent drawn uniformly among the
                 earlier bodies, placed at the sum of the two mean half-extents along a random
                 direction.
"""
import math

import numpy as np

from . import motors_np
from .abi import (BODY_DTYPE, GRAVITY_OFF, GRAVITY_PLUMMER, JOINT_DTYPE, LIE_EULER, NEWTON, PRECISION_F64,
                  step_params)

IDENTITY = np.array([1.0, 0, 0, 0, 0, 0, 0, 0])


def translation(x):
    return motors_np.twist_exp_n(np.array([x[0], x[1], x[2], 0.0, 0.0, 0.0]), 1.0)[0]


def random_unit(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def gravity_world(n, radius=100.0, seed=0, G=1.0):
    """Point masses with circular-orbit velocities (isotropic unit moment, as
    RigidBody::body_at_with_speed_and_mass, crates/newton/src/body.rs:104-128)."""
    rng = np.random.default_rng(seed)
    u = rng.random(n)
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    pos = dirs * (radius * np.cbrt(u))[:, None]
    mass = np.exp(rng.uniform(math.log(1.0), math.log(10.0), size=n))
    com = (mass[:, None] * pos).sum(0) / mass.sum()
    rel = pos - com
    r = np.linalg.norm(rel, axis=1)
    order = np.argsort(r, kind="stable")
    enclosed = np.zeros(n)
    # mass strictly inside each body's radius (ties at equal radius excluded)
    sorted_r = r[order]
    first_idx = np.searchsorted(sorted_r, sorted_r, side="left")
    enclosed[order] = np.concatenate([[0.0], np.cumsum(mass[order])])[first_idx]
    safe_r = np.where(r > 0.0, r, 1.0)
    rhat = rel / safe_r[:, None]
    t = np.cross(np.array([0.0, 0.0, 1.0]), rhat)
    tn = np.linalg.norm(t, axis=1)
    par = tn < 1e-12
    if par.any():
        ax = rng.normal(size=(int(par.sum()), 3))
        t[par] = np.cross(ax / np.linalg.norm(ax, axis=1, keepdims=True), rhat[par])
        tn = np.linalg.norm(t, axis=1)
    t /= np.where(tn > 0, tn, 1.0)[:, None]
    speed = np.sqrt(G * enclosed / safe_r)
    vel = np.where((r > 0.0)[:, None], speed[:, None] * t, 0.0)
    vel += rng.normal(0.0, 0.01, size=(n, 3))
    bodies = np.zeros(n, dtype=BODY_DTYPE)
    tw = np.zeros((n, 6))
    tw[:, :3] = pos
    bodies["pose"] = motors_np.twist_exp_n(tw, 1.0)
    bodies["momentum"][:, :3] = mass[:, None] * vel
    bodies["mass"] = mass
    bodies["inertia"][:, 0] = 1.0
    bodies["inertia"][:, 4] = 1.0
    bodies["inertia"][:, 8] = 1.0
    bodies["diagonal"] = 1
    bodies["size"] = np.cbrt(mass / 4.0)
    return bodies


def _boxes(rng, n):
    h = rng.uniform(0.5, 2.0, size=(n, 3))
    mass = 8.0 * h[:, 0] * h[:, 1] * h[:, 2]
    I = np.zeros((n, 9))
    I[:, 0] = mass / 3.0 * (h[:, 1] ** 2 + h[:, 2] ** 2)
    I[:, 4] = mass / 3.0 * (h[:, 0] ** 2 + h[:, 2] ** 2)
    I[:, 8] = mass / 3.0 * (h[:, 0] ** 2 + h[:, 1] ** 2)
    return h, mass, I


def _edge_joints(rng, a, b, rest, laws):
    """Per edge (a[e], b[e]): the axial spring-damper then the dampers, edge by edge."""
    ne = len(a)
    k = np.exp(rng.uniform(math.log(1e2), math.log(1e4), size=ne))
    c = 0.1 * np.sqrt(k)
    per = len(laws)
    j = np.zeros(ne * per, dtype=JOINT_DTYPE)
    for slot, law in enumerate(laws):
        sel = j[slot::per]
        sel["law"] = law
        sel["a"] = a
        sel["b"] = b
        if law <= 1:
            sel["params"][:, 6] = rest
            sel["params"][:, 7] = k
            sel["params"][:, 8] = c
            sel["params"][:, 9] = 1e-6
        elif law == 2:
            sel["params"][:, 0] = c
            sel["params"][:, 1] = 1e-6
        else:
            sel["params"][:, 0] = c
        j[slot::per] = sel
    return j


def _bodies_at(rng, mass, I, pos, twist_sigma):
    n = len(mass)
    bodies = np.zeros(n, dtype=BODY_DTYPE)
    bodies["mass"] = mass
    bodies["inertia"] = I
    bodies["diagonal"] = 1
    bodies["size"] = np.cbrt(mass / 4.0)
    xi = rng.normal(0.0, twist_sigma, size=(n, 6))
    tw = np.zeros((n, 6))
    tw[:, :3] = pos
    bodies["pose"] = motors_np.compose_n(motors_np.twist_exp_n(xi, 1.0), motors_np.twist_exp_n(tw, 1.0))
    return bodies


def chain_world(n, seed=1, origin=(0.0, 0.0, 0.0), twist_sigma=0.05, laws=(0, 2, 3)):
    rng = np.random.default_rng(seed)
    h, mass, I = _boxes(rng, n)
    x = np.concatenate([[0.0], np.cumsum(h[:-1, 0] + h[1:, 0])])
    x -= x.mean()
    pos = np.zeros((n, 3))
    pos[:, 0] = x
    pos += np.asarray(origin, dtype=np.float64)
    joints = _edge_joints(rng, np.arange(n - 1), np.arange(1, n), x[1:] - x[:-1], laws)
    return _bodies_at(rng, mass, I, pos, twist_sigma), joints


def tree_world(n, seed=2, twist_sigma=0.05, laws=(0, 2, 3)):
    rng = np.random.default_rng(seed)
    h, mass, I = _boxes(rng, n)
    rad = h.mean(axis=1)
    parent = np.zeros(n, dtype=np.int64)
    if n > 1:
        parent[1:] = np.floor(rng.random(n - 1) * np.arange(1, n)).astype(np.int64)
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    dist = rad[parent] + rad
    pos = np.zeros((n, 3))
    done = np.zeros(n, dtype=bool)
    done[0] = True
    while not done.all():  # resolve level by level: a node's parent precedes it
        ready = (~done) & done[parent]
        pos[ready] = pos[parent[ready]] + dist[ready, None] * dirs[ready]
        done |= ready
    pos -= (mass[:, None] * pos).sum(0) / mass.sum()
    child = np.arange(1, n)
    joints = _edge_joints(rng, parent[1:], child, dist[1:], laws)
    return _bodies_at(rng, mass, I, pos, twist_sigma), joints


def cloth_world(cols, rows, kick=0.5, k=100.0, zeta=0.7, mass_total=1.0, width=0.5, g=9.81, wind=1.0, dt=1.0 / 60.0,
                tol=1e-4, precision=PRECISION_F64):
    """The reference's curtain (crates/newton/tests/cloth_grid_stability.rs:48-110,
    cloth_scaling.rs:40-90): a cols x rows grid in the XZ plane with spacing h = width / (cols - 1),
    the top row kinematic at rest, every other node a point body of mass mass_total / (cols rows)
    with unit isotropic moment; nodes whose row-major index is 1 mod 4 start at kick along +Y. An
    axial SimpleSpringDamper (anchors at the centres, rest h, stiffness k, damping
    zeta 2 sqrt(k m / 2), softening 1e-6) joins each node to its right and its upper neighbour, in
    row-major order, right before up. Gravity -g along Z and a wind of `wind` along Y act as
    uniform fields. The grid's springs close cycles among the dynamic bodies."""
    h = width / (cols - 1.0)
    m = mass_total / (cols * rows)
    c = zeta * 2.0 * math.sqrt(k * (m * 0.5))
    n = cols * rows
    bodies = np.zeros(n, dtype=BODY_DTYPE)
    tw = np.zeros((n, 6))
    for row in range(rows):
        for col in range(cols):
            i = row * cols + col
            tw[i, :3] = (col * h, 0.0, row * h)
    bodies["pose"] = motors_np.twist_exp_n(tw, 1.0)
    bodies["inertia"][:, 0] = bodies["inertia"][:, 4] = bodies["inertia"][:, 8] = 1.0
    bodies["diagonal"] = 1
    top = np.arange(n) >= (rows - 1) * cols
    bodies["kinematic"] = top.astype(np.int32)
    bodies["mass"] = np.where(top, 0.0, m)
    bodies["size"] = np.cbrt(m / 4.0)
    gust = (~top) & (np.arange(n) % 4 == 1)
    bodies["momentum"][gust, 1] = m * kick
    edges = []
    for row in range(rows):
        for col in range(cols):
            i = row * cols + col
            if col + 1 < cols:
                edges.append((i, i + 1))
            if row + 1 < rows:
                edges.append((i, i + cols))
    joints = np.zeros(len(edges), dtype=JOINT_DTYPE)
    for q, (a, b) in enumerate(edges):
        joints[q]["law"], joints[q]["a"], joints[q]["b"] = 0, a, b
        joints[q]["params"][6:10] = (h, k, c, 1e-6)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=dt, tol=tol,
                         field=(0.0, wind, -g))
    return bodies, joints, params


def camera_rig_world(n_rigs=1, r_object=2.0, linear=1.0, spacing=1000.0, dt=1.0 / 60.0, tol=1e-10,
                     precision=PRECISION_F64, target_velocity=(0.0, 0.0, 0.0)):
    """The hitchcock camera rig (crates/hitchcock/src/camera.rs:259-520, rig.rs:86-147) as a
    consumer workload: per rig four bodies, in this order, the eye (`real`, at the target's
    centre + r along z), the `intermediate` (at the centre) and the `anchor` (centre - r along y),
    each a unit mass with unit isotropic moment moving with the target's velocity
    (RigidBody::body_at_with_speed_and_mass), and the kinematic target tracker at the centre; 17
    CriticallyDampedWarped axial springs between offset anchors (stiffness `linear`, softening
    r / 1000, the rests of camera.rs:345-489: 0, 0, r sqrt2, r sqrt2 eye-intermediate; r sqrt2 x 8
    intermediate-tracker; r x 4 intermediate-anchor; r anchor-tracker), three TorsionalDamperWarped
    (eye-intermediate, intermediate-anchor, intermediate-tracker) and two PerpendicularDamperWarped
    (intermediate-tracker, anchor-tracker), each with damping `linear`, connected in that order.
    Rig k's target starts at (spacing k, 0, 0). The host moves each tracker between steps
    (camera.rs:55-76: pose = translation to the target, momentum = the target's velocity), see
    track_targets. Gravity off; implicit Newton."""
    r, z = float(r_object), 0.0
    s1 = r * math.sqrt(2.0)
    soft = r / 1000.0
    springs = [  # (a, a_local, b, b_local, rest) with 0 eye, 1 intermediate, 2 anchor, 3 tracker
        (0, (r, z, -r), 1, (r, z, z), z), (0, (-r, z, -r), 1, (-r, z, z), z),
        (0, (z, r, z), 1, (z, z, z), s1), (0, (z, -r, z), 1, (z, z, z), s1),
        (1, (r, -r, z), 3, (z, z, z), s1), (1, (-r, -r, z), 3, (z, z, z), s1),
        (1, (z, -r, -r), 3, (z, z, z), s1), (1, (z, -r, r), 3, (z, z, z), s1),
        (1, (r, r, z), 3, (z, z, z), s1), (1, (-r, r, z), 3, (z, z, z), s1),
        (1, (z, r, -r), 3, (z, z, z), s1), (1, (z, r, r), 3, (z, z, z), s1),
        (1, (r, -r, z), 2, (z, z, z), r), (1, (-r, -r, z), 2, (z, z, z), r),
        (1, (z, -r, -r), 2, (z, z, z), r), (1, (z, -r, r), 2, (z, z, z), r),
        (2, (z, z, z), 3, (z, z, z), r),
    ]
    torsional = [(0, 1), (1, 2), (1, 3)]
    transverse = [(1, 3), (2, 3)]
    nb, nj = 4 * n_rigs, (len(springs) + len(torsional) + len(transverse)) * n_rigs
    bodies = np.zeros(nb, dtype=BODY_DTYPE)
    joints = np.zeros(nj, dtype=JOINT_DTYPE)
    tw = np.zeros((nb, 6))
    v = np.asarray(target_velocity, dtype=np.float64)
    q = 0
    for k in range(n_rigs):
        c = np.array([spacing * k, 0.0, 0.0])
        o = 4 * k
        for i, off in enumerate(((z, z, r), (z, z, z), (z, -r, z), (z, z, z))):
            tw[o + i, :3] = c + np.array(off)
        for i in range(3):
            bodies[o + i]["mass"] = 1.0
            bodies[o + i]["momentum"][:3] = v
        bodies[o + 3]["kinematic"] = 1
        bodies[o + 3]["mass"] = 0.0
        bodies[o + 3]["momentum"][:3] = v  # Inertia::Kinematic: the momentum is the twist
        for a, al, b, bl, rest in springs:
            joints[q]["law"], joints[q]["a"], joints[q]["b"] = 1, o + a, o + b
            joints[q]["params"][:10] = (*al, *bl, rest, linear, 0.0, soft)
            q += 1
        for a, b in torsional:
            joints[q]["law"], joints[q]["a"], joints[q]["b"] = 3, o + a, o + b
            joints[q]["params"][0] = linear
            q += 1
        for a, b in transverse:
            joints[q]["law"], joints[q]["a"], joints[q]["b"] = 2, o + a, o + b
            joints[q]["params"][:2] = (linear, soft)
            q += 1
    bodies["pose"] = motors_np.twist_exp_n(tw, 1.0)
    bodies["inertia"][:, 0] = bodies["inertia"][:, 4] = bodies["inertia"][:, 8] = 1.0
    bodies["diagonal"] = 1
    bodies["size"] = 1.0
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=dt, tol=tol)
    return bodies, joints, params


def track_targets(state, n_rigs, centres, velocities):
    """The tracker's pre_step (crates/hitchcock/src/camera.rs:55-76) on an (n, 14) state array
    (pose, momentum per body, as exg_world_get_state returns it): tracker k (body 4k + 3) moves to
    centres[k] with velocity velocities[k]."""
    out = state.copy()
    tw = np.zeros((n_rigs, 6))
    tw[:, :3] = centres
    out[3::4, :8] = motors_np.twist_exp_n(tw, 1.0)
    out[3::4, 8:11] = velocities
    out[3::4, 11:14] = 0.0
    return out


def concat_worlds(parts):
    """Concatenate (bodies, joints) pairs into one world, re-indexing the joints."""
    bodies, joints, off = [], [], 0
    for b, j in parts:
        bodies.append(b)
        jj = j.copy()
        jj["a"] += off
        jj["b"] += off
        joints.append(jj)
        off += len(b)
    return np.concatenate(bodies), (np.concatenate(joints) if joints else np.zeros(0, dtype=JOINT_DTYPE))


# ── the configurations (sizes as stated; `scale` shrinks them for quick checks only) ──
def config0(seed=0):
    """1024 point masses, ball radius 100, Plummer eps 0.05, LieEuler, dt 1e-3, 1000 steps."""
    bodies = gravity_world(1024, 100.0, seed)
    params = step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=PRECISION_F64, G=1.0,
                         softening=0.05, dt=1e-3)
    return bodies, np.zeros(0, dtype=JOINT_DTYPE), params, 1000


def config1(seed=1, n=256):
    """Serial chain of 256 boxes, implicit Newton, tol 1e-10, dt 1e-2, 500 steps, gravity off."""
    bodies, joints = chain_world(n, seed)
    params = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=PRECISION_F64, dt=1e-2, tol=1e-10)
    return bodies, joints, params, 500


def config2_parts(seed=2, n_gravity=65536, n_chains=16, chain_len=256, precision=PRECISION_F64, exact_jacobian=False):
    """65,536 gravity bodies (ball radius 1000) and 16 independent 256-body chains, stepped together at
    dt 1e-3 for 1000 steps; returned as (gravity world, chain world) parts of one epoch."""
    g = gravity_world(n_gravity, 1000.0, seed)
    gparams = step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=precision, G=1.0,
                          softening=0.05, dt=1e-3)
    chains = [chain_world(chain_len, seed * 1000 + c, origin=(0.0, 50.0 * c, 5000.0)) for c in range(n_chains)]
    cb, cj = concat_worlds(chains)
    cparams = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=1e-3, tol=1e-10,
                          exact_jacobian=exact_jacobian)
    return (g, np.zeros(0, dtype=JOINT_DTYPE), gparams), (cb, cj, cparams), 1000


def config3_sizes(n_worlds=4096, seed=3, lo=8, hi=8192):
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_worlds))).astype(np.int64)


def config3_worlds(n_worlds=4096, seed=3, precision=PRECISION_F64, lo=8, hi=8192, exact_jacobian=False, only=None):
    """4096 independent worlds, body counts log-uniform in [8, 8192]: even-numbered worlds are
    gravity worlds (config 0 distributions, LieEuler, dt 1e-3), odd-numbered ones are random
    trees (config 1 laws and parameters, implicit Newton tol 1e-10, dt 1e-2). `only` keeps a
    subset of the world indices (each world's content depends on its index alone)."""
    sizes = config3_sizes(n_worlds, seed, lo, hi)
    gp = step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=precision, G=1.0, softening=0.05,
                     dt=1e-3)
    tp = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=1e-2, tol=1e-10,
                     exact_jacobian=exact_jacobian)
    worlds = []
    keep = None if only is None else set(only)
    for k, n in enumerate(sizes):
        if keep is not None and k not in keep:  # a rank's share: the same worlds, the others skipped
            continue
        if k % 2 == 0:
            worlds.append((gravity_world(int(n), 100.0, seed * 100003 + k), np.zeros(0, dtype=JOINT_DTYPE), gp))
        else:
            b, j = tree_world(int(n), seed * 100003 + k)
            worlds.append((b, j, tp))
    return worlds
