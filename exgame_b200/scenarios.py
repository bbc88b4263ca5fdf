"""Seeded synthetic workloads (the reference ships no benchmark data; these stand in for the
configurations the measurements are quoted on).

Every generator draws from numpy's PCG64 (`numpy.random.default_rng(seed)`) and returns host
arrays in the C ABI's record layouts (BODY_DTYPE, JOINT_DTYPE) plus step parameters. Motors are
built with the library's own host-side algebra (exg_motor_exp / exg_motor_compose).

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

from . import _lib
from .abi import (BODY_DTYPE, GRAVITY_OFF, GRAVITY_PLUMMER, JOINT_DTYPE, LIE_EULER, NEWTON, PRECISION_F64,
                  step_params)

IDENTITY = np.array([1.0, 0, 0, 0, 0, 0, 0, 0])


def translation(x):
    return _lib.motor_exp(np.array([x[0], x[1], x[2], 0.0, 0.0, 0.0]), 1.0)


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
    vel = np.zeros((n, 3))
    zhat = np.array([0.0, 0.0, 1.0])
    for i in range(n):
        if r[i] == 0.0:
            continue
        rhat = rel[i] / r[i]
        t = np.cross(zhat, rhat)
        if np.linalg.norm(t) < 1e-12:
            t = np.cross(random_unit(rng), rhat)
        t /= np.linalg.norm(t)
        vel[i] = math.sqrt(G * enclosed[i] / r[i]) * t
    vel += rng.normal(0.0, 0.01, size=(n, 3))
    bodies = np.zeros(n, dtype=BODY_DTYPE)
    for i in range(n):
        bodies[i]["pose"] = translation(pos[i])
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


def _joint_triplet(rng, a, b, rest, laws):
    k = math.exp(rng.uniform(math.log(1e2), math.log(1e4)))
    c = 0.1 * math.sqrt(k)
    out = []
    axial = np.zeros((), dtype=JOINT_DTYPE)
    axial["law"], axial["a"], axial["b"] = laws[0], a, b
    axial["params"][:10] = [0, 0, 0, 0, 0, 0, rest, k, c, 1e-6]
    out.append(axial)
    if len(laws) > 1:
        perp = np.zeros((), dtype=JOINT_DTYPE)
        perp["law"], perp["a"], perp["b"] = laws[1], a, b
        perp["params"][:2] = [c, 1e-6]
        out.append(perp)
    if len(laws) > 2:
        tors = np.zeros((), dtype=JOINT_DTYPE)
        tors["law"], tors["a"], tors["b"] = laws[2], a, b
        tors["params"][0] = c
        out.append(tors)
    return out


def _place(rng, bodies, pos, twist_sigma):
    for i in range(len(bodies)):
        xi = rng.normal(0.0, twist_sigma, size=6)
        bodies[i]["pose"] = _lib.motor_compose(_lib.motor_exp(xi, 1.0), translation(pos[i]))


def chain_world(n, seed=1, origin=(0.0, 0.0, 0.0), twist_sigma=0.05, laws=(0, 2, 3)):
    rng = np.random.default_rng(seed)
    h, mass, I = _boxes(rng, n)
    x = np.zeros(n)
    for i in range(1, n):
        x[i] = x[i - 1] + h[i - 1, 0] + h[i, 0]
    x -= x.mean()
    pos = np.zeros((n, 3))
    pos[:, 0] = x
    pos += np.asarray(origin, dtype=np.float64)
    bodies = np.zeros(n, dtype=BODY_DTYPE)
    bodies["mass"] = mass
    bodies["inertia"] = I
    bodies["diagonal"] = 1
    bodies["size"] = np.cbrt(mass / 4.0)
    joints = []
    for i in range(n - 1):
        joints += _joint_triplet(rng, i, i + 1, x[i + 1] - x[i], laws)
    _place(rng, bodies, pos, twist_sigma)
    return bodies, np.array(joints, dtype=JOINT_DTYPE)


def tree_world(n, seed=2, twist_sigma=0.05, laws=(0, 2, 3)):
    rng = np.random.default_rng(seed)
    h, mass, I = _boxes(rng, n)
    rad = h.mean(axis=1)
    pos = np.zeros((n, 3))
    joints = []
    for i in range(1, n):
        p = int(rng.integers(0, i))
        d = rad[p] + rad[i]
        pos[i] = pos[p] + d * random_unit(rng)
        joints += _joint_triplet(rng, p, i, d, laws)
    pos -= (mass[:, None] * pos).sum(0) / mass.sum()
    bodies = np.zeros(n, dtype=BODY_DTYPE)
    bodies["mass"] = mass
    bodies["inertia"] = I
    bodies["diagonal"] = 1
    bodies["size"] = np.cbrt(mass / 4.0)
    _place(rng, bodies, pos, twist_sigma)
    return bodies, np.array(joints, dtype=JOINT_DTYPE)


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


def config2_parts(seed=2, n_gravity=65536, n_chains=16, chain_len=256, precision=PRECISION_F64):
    """65,536 gravity bodies (ball radius 1000) and 16 independent 256-body chains, stepped together at
    dt 1e-3 for 1000 steps; returned as (gravity world, chain world) parts of one epoch."""
    g = gravity_world(n_gravity, 1000.0, seed)
    gparams = step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=precision, G=1.0,
                          softening=0.05, dt=1e-3)
    chains = [chain_world(chain_len, seed * 1000 + c, origin=(0.0, 50.0 * c, 5000.0)) for c in range(n_chains)]
    cb, cj = concat_worlds(chains)
    cparams = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, precision=precision, dt=1e-3, tol=1e-10)
    return (g, np.zeros(0, dtype=JOINT_DTYPE), gparams), (cb, cj, cparams), 1000


def config3_sizes(n_worlds=4096, seed=3, lo=8, hi=8192):
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), size=n_worlds))).astype(np.int64)
