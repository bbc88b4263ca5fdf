"""Pins the oracle to the reference's own known answers and test properties.

The reference stores no golden vectors; every case here restates an assertion of its test suite
(file:line cited per test) and checks the f64 restatement against it. These run on the CPU.
"""
import ctypes

import numpy as np
import pytest

from exgame_b200 import scenarios
from exgame_b200.abi import (BODY_DTYPE, GRAVITY_OFF, GRAVITY_PLUMMER, GRAVITY_SIZE_CORE, JOINT_DTYPE, LIE_EULER,
                             NEWTON, EXPLICIT_EULER, SYMPLECTIC_EULER, step_params)


def body(pos=(0, 0, 0), vel=(0, 0, 0), mass=1.0, moments=(1.0, 1.0, 1.0), kinematic=False, oracle=None):
    b = np.zeros((), dtype=BODY_DTYPE)
    b["pose"] = scenarios.translation(np.asarray(pos, float))
    b["momentum"][:3] = np.asarray(vel, float) * (1.0 if kinematic else mass)
    b["mass"] = 0.0 if kinematic else mass
    b["inertia"][[0, 4, 8]] = moments
    b["diagonal"] = 1
    b["kinematic"] = int(kinematic)
    b["size"] = (mass / 4.0) ** (1.0 / 3.0) if not kinematic else 1.0
    return b


def spring(a, b, rest, k, c, law=0):
    j = np.zeros((), dtype=JOINT_DTYPE)
    j["law"], j["a"], j["b"] = law, a, b
    j["params"][:10] = [0, 0, 0, 0, 0, 0, rest, k, c, 1e-6]
    return j


def position(b):
    from exgame_b200 import _lib
    return _lib.motor_apply_point(b["pose"], np.zeros(3))


# ── algebra: the sign law and the derived markup (crates/clifford/src/algebra/mod.rs) ──
def test_degenerate_generator_annihilates(oracle):
    L = oracle.lib()
    s, m = ctypes.c_int(), ctypes.c_int()
    L.orc_blade_prod(0b1000, 0b1000, ctypes.byref(s), ctypes.byref(m))
    assert s.value == 0  # e0^2 = 0 (mod.rs:187-195)
    L.orc_blade_prod(0b1000, 0b0001, ctypes.byref(s), ctypes.byref(m))
    assert m.value == 0b1001 and s.value != 0


def test_orientation_anchor_every_blade(oracle):
    # b ^ dual(b) = +I for every blade (mod.rs:145-158, 200-220)
    L = oracle.lib()
    for b in range(16):
        comp = 15 ^ b
        s, m = ctypes.c_int(), ctypes.c_int()
        L.orc_blade_prod(b, comp, ctypes.byref(s), ctypes.byref(m))
        assert m.value == 15
        inv = sum(bin(comp & ((1 << bi) - 1)).count("1") for bi in range(4) if (b >> bi) & 1)
        assert s.value * (1 if inv % 2 == 0 else -1) == 1


def test_twist_components_roundtrip_and_rotations(oracle):
    # motor.rs:330-404: +90 deg about z, 180 deg, translation, dt scales the angle
    def apply(m, p):
        o = np.zeros(3)
        oracle.lib().orc_motor_apply_point(oracle.p(m), oracle.p(oracle.arr(p)), oracle.p(o))
        return o
    assert np.allclose(apply(oracle.twist_exp([0, 0, 0, 0, 0, np.pi / 2]), [1, 0, 0]), [0, 1, 0], atol=1e-9)
    assert np.allclose(apply(oracle.twist_exp([0, 0, 0, 0, 0, np.pi]), [1, 0, 0]), [-1, 0, 0], atol=1e-9)
    assert np.allclose(apply(oracle.twist_exp([0, 0, 0, 0, 0, np.pi / 2], 2.0), [1, 0, 0]), [-1, 0, 0], atol=1e-9)
    assert np.allclose(apply(oracle.twist_exp([2, 0, 0, 0, 0, 0]), [0, 0, 0]), [2, 0, 0], atol=1e-12)
    # rotor is unit: <M M~>_0 = 1 (motor.rs:430-437): M * M^-1 = identity
    m = oracle.twist_exp([0, 0, 0, 0.3, -0.2, 0.5])
    inv = np.zeros(8)
    oracle.lib().orc_motor_inverse(oracle.p(m), oracle.p(inv))
    prod = np.zeros(8)
    oracle.lib().orc_motor_compose(oracle.p(m), oracle.p(inv), oracle.p(prod))
    assert np.allclose(prod, [1, 0, 0, 0, 0, 0, 0, 0], atol=1e-12)


def test_power_invariant_under_transport(oracle):
    # screw.rs:455-475: <coAd(w), Ad(t)> == <w, t>
    L = oracle.lib()
    w = oracle.arr([2.0, -1.0, 0.5, 0.3, 0.8, -0.4])
    t = oracle.arr([1.0, 2.0, 3.0, 0.5, -1.0, 0.7])
    m = oracle.twist_exp([0.3, -0.2, 0.5, 0.1, 0.4, -0.2])
    wt, tt = np.zeros(6), np.zeros(6)
    L.orc_twist_transport(oracle.p(w), oracle.p(m), 1, oracle.p(wt))
    L.orc_twist_transport(oracle.p(t), oracle.p(m), 0, oracle.p(tt))
    assert abs(L.orc_power(oracle.p(w), oracle.p(t)) - L.orc_power(oracle.p(wt), oracle.p(tt))) < 1e-9
    # power = f.v + tau.w
    assert abs(L.orc_power(oracle.p(w), oracle.p(t)) - (w[:3] @ t[:3] + w[3:] @ t[3:])) < 1e-12
    assert not np.allclose(wt, tt)  # the two laws differ


def test_velocity_at_is_omega_cross_r(oracle):
    # the angular markup is solved from velocity = omega x r (markup.rs:53-82)
    v = np.zeros(3)
    oracle.lib().orc_velocity_at(oracle.p(oracle.arr([0, 0, 0, 0, 0, 1])), oracle.p(oracle.arr([1, 0, 0])), oracle.p(v))
    assert np.allclose(v, [0, 1, 0])


def test_study_forms_agree_across_the_seam(oracle):
    # crates/peano/src/scalar.rs:199-347: both arms agree at the seam, 1e-13 (f64), 1e-6 (f32)
    L = oracle.lib()
    for u in (0.9e-9, 1.1e-9, 1e-6, 1e-4, 0.5):
        o = np.zeros(3)
        L.orc_study_forms(ctypes.c_double(u), oracle.p(o))
        l = np.sqrt(u)
        assert abs(o[0] - np.sin(l) / l) < 1e-13
        assert abs(o[1] - np.cos(l)) < 1e-13
    o = np.zeros(3)
    L.orc_study_forms(ctypes.c_double(0.0), oracle.p(o))
    assert o[0] == 1.0 and o[1] == 1.0 and o[2] == -1.0 / 6.0
    of = np.zeros(3, dtype=np.float32)
    for u in (0.9e-5, 1.1e-5):
        L.orc_study_forms_f32(ctypes.c_float(u), ctypes.c_void_p(of.ctypes.data))
        l = np.sqrt(u)
        assert abs(of[0] - np.sin(l) / l) < 1e-6


# ── gravity (crates/newton/src/gravity.rs) ───────────────────────────────────
def test_pair_force_inverse_square(oracle):
    # gravity.rs:722-738: g = 2, d = 3 -> F/g = 2/9 toward +x
    o = np.zeros(3)
    ok = oracle.lib().orc_pair_force_literal(oracle.p(np.zeros(3)), 2.0, oracle.p(oracle.arr([3, 0, 0])), 2.0, 1.0,
                                            oracle.p(o))
    assert ok == 1
    assert abs(o[0] / 2.0 - 2.0 / 9.0) < 1e-12 and abs(o[1]) < 1e-15 and abs(o[2]) < 1e-15


def test_pair_force_coincident_is_none(oracle):
    # gravity.rs:740-750
    o = np.zeros(3)
    pt = oracle.arr([1, 2, 3])
    assert oracle.lib().orc_pair_force_literal(oracle.p(pt), 1.0, oracle.p(pt), 1.0, 1.0, oracle.p(o)) == 0


def test_pair_force_literal_matches_closed_form(oracle):
    rng = np.random.default_rng(1)
    for _ in range(50):
        a, b = rng.normal(size=3) * 3, rng.normal(size=3) * 3
        ga, gb, size = rng.uniform(1, 5), rng.uniform(1, 5), rng.uniform(0.5, 2.0)
        o = np.zeros(3)
        oracle.lib().orc_pair_force_literal(oracle.p(a), ga, oracle.p(b), gb, size, oracle.p(o))
        d = np.linalg.norm(b - a)
        core = max(d, size)
        assert np.allclose(o, ga * gb * (b - a) / core ** 3, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("law", [GRAVITY_SIZE_CORE, GRAVITY_PLUMMER])
def test_third_law_two_and_three_bodies(oracle, law):
    # gravity.rs:780-904: total wrench of the pair / triple is zero
    for n in (2, 3):
        bs = np.array([body(p, mass=m) for p, m in zip([(-1, 0, 0), (1, 0, 0), (0, 2, 0.5)], (1.0, 2.0, 3.0))][:n])
        f = oracle.gravity_forces(bs, law, 1.0, 0.05)
        assert np.allclose(f.sum(0), 0.0, atol=1e-14)
        assert f[0][0] > 0  # attraction toward +x


# ── joint laws (crates/joints) ─────────────────────────────────────────────────
KDO_POSE_A = [0.5, -0.3, 0.2, 0.1, 0.4, -0.2]   # crates/viete/tests/kernel_differential_oracle.rs:160-179
KDO_POSE_B = [-0.4, 0.25, 0.15, 0.2, -0.1, 0.3]
KDO_VA = [0.40, -0.20, 0.35, 0.12, -0.28, 0.18]
KDO_VB = [-0.30, 0.45, -0.15, 0.22, 0.14, -0.26]
KDO_PARAMS = [0.3, -0.2, 0.15, -0.1, 0.25, -0.05, 1.3, 7.0, 2.0, 1e-6]


def test_kernel_differential_fixed_point_is_densely_coupled(oracle):
    # kernel_differential_oracle.rs:155-261: CriticallyDampedWarped at the fixed point, >= 250/300 nonzero
    pa, pb = oracle.twist_exp(KDO_POSE_A), oracle.twist_exp(KDO_POSE_B)
    J = oracle.jacobian_eval(1, KDO_PARAMS, pa, pb, KDO_VA, KDO_VB, 0.016, 1.3)
    assert (np.abs(J) > 1e-9).sum() >= 250
    plain = oracle.plain_eval(1, KDO_PARAMS, pa, pb, KDO_VA, KDO_VB, 0.016, 1.3)
    assert np.array_equal(plain, J[:, 0])  # value of the Jacobian kernel == plain kernel (accelerator/mod.rs:1410-1492)


@pytest.mark.parametrize("law", [0, 1, 2, 3])
def test_jacobian_matches_finite_differences(oracle, law):
    """AD Jacobian vs central differences along each of the 24 axes (pose axes perturb by
    exp(h e_k) * pose, velocity axes additively)."""
    pa, pb = oracle.twist_exp(KDO_POSE_A), oracle.twist_exp(KDO_POSE_B)
    prm = list(KDO_PARAMS) if law <= 1 else ([2.0, 1e-3] + [0] * 8 if law == 2 else [1.5] + [0] * 9)
    J = oracle.jacobian_eval(law, prm, pa, pb, KDO_VA, KDO_VB, 0.016, 1.3)
    h = 1e-6
    for k in range(24):
        def ev(sign):
            qa, qb, va, vb = pa.copy(), pb.copy(), np.array(KDO_VA), np.array(KDO_VB)
            if k < 12:
                e = np.zeros(6)
                e[k % 6] = sign * h
                # exp(delta) with the unit retraction = Twist::exp(2 delta)
                d = oracle.twist_exp(e, 2.0)
                out = np.zeros(8)
                tgt = qa if k < 6 else qb
                oracle.lib().orc_motor_compose(oracle.p(tgt), oracle.p(d), oracle.p(out))
                if k < 6:
                    qa = out
                else:
                    qb = out
            elif k < 18:
                va[k - 12] += sign * h
            else:
                vb[k - 18] += sign * h
            return oracle.plain_eval(law, prm, qa, qb, va, vb, 0.016, 1.3)
        fd = (ev(1) - ev(-1)) / (2 * h)
        assert np.allclose(J[:, 1 + k], fd, rtol=1e-5, atol=1e-6), (law, k)


def test_perpendicular_damper_reaction_cancels_and_dissipates(oracle):
    # perpendicular_damper_warped.rs:198-292
    rng = np.random.default_rng(7)
    for _ in range(20):
        pa = oracle.twist_exp(np.r_[rng.normal(size=3) * 2, rng.normal(size=3) * 0.5])
        pb = oracle.twist_exp(np.r_[rng.normal(size=3) * 2, rng.normal(size=3) * 0.5])
        va, vb = rng.normal(size=6), rng.normal(size=6)
        w = oracle.plain_eval(2, [1.0, 1e-3] + [0] * 8, pa, pb, va, vb, 1 / 60, 1.0)
        assert np.allclose(w[:6] + w[6:], 0.0, atol=1e-15)
        L = oracle.lib()
        pw = L.orc_power(oracle.p(w[:6].copy()), oracle.p(oracle.arr(va))) + \
            L.orc_power(oracle.p(w[6:].copy()), oracle.p(oracle.arr(vb)))
        assert pw <= 1e-12


def test_critically_damped_is_tension_positive(oracle):
    # critically_damped_warped.rs:101-122: dt = 0, warp = 1, stretched -> attraction on a toward b
    pa, pb = scenarios.translation([0, 0, 0]), scenarios.translation([4, 0, 0])
    z = [0.0] * 6
    for law in (0, 1):
        w = oracle.plain_eval(law, [0, 0, 0, 0, 0, 0, 2.0, 10.0, 0.0, 1e-6], pa, pb, z, z, 0.0, 1.0)
        assert w[0] > 0  # force on a points toward b (+x): tension


def test_params_flatten_order():
    # crates/joints/src/lib.rs:273-298: [a0,a1,a2, b0,b1,b2, rest, k, c, soft]
    j = spring(0, 1, 1.3, 7.0, 2.0)
    assert list(j["params"][6:10]) == [1.3, 7.0, 2.0, 1e-6]


# ── integrators ─────────────────────────────────────────────────────────────────
def world_momentum_drift(oracle, integrator, dt, steps):
    b = body(moments=(2.0, 3.0, 4.0))
    b["momentum"][3:] = [2.0 * 1.0, 3.0 * 1.5, 4.0 * 0.7]
    w = oracle.OracleWorld(np.array([b]), np.zeros(0, dtype=JOINT_DTYPE), step_params(integrator=integrator, dt=dt))
    from exgame_b200 import _lib
    l0 = _lib.screw_transport(w.bodies()[0]["momentum"], w.bodies()[0]["pose"], 1)[3:]
    w.step(steps)
    bb = w.bodies()[0]
    l1 = _lib.screw_transport(bb["momentum"], bb["pose"], 1)[3:]
    return np.linalg.norm(l1 - l0)


def test_lie_euler_conserves_world_momentum(oracle):
    # lie_euler.rs:64-100 (f32 bound 1e-3; here f64)
    assert world_momentum_drift(oracle, LIE_EULER, 0.01, 2000) < 1e-9


def test_lie_world_momentum_independent_of_dt(oracle):
    # lie_euler.rs:104-114: coarse (dt 0.01, 200 steps) and fine (dt 0.0005, 4000 steps) both stay
    # at round-off (f32 bounds 1e-4 and 1e-2 there; f64 here)
    coarse = world_momentum_drift(oracle, LIE_EULER, 0.01, 200)
    fine = world_momentum_drift(oracle, LIE_EULER, 0.0005, 4000)
    assert coarse < 1e-4 and fine < 1e-2
    assert coarse < 1e-11 and fine < 1e-10, (coarse, fine)


def test_lie_off_axis_spinning_body_keeps_com_in_place(oracle):
    # lie_euler.rs:116-160: a body at x = 10 spinning about its own z axis (isotropic 0.4, omega_z 1)
    # keeps its centre of mass over 100 steps of 0.01: the body-frame increment composes on the
    # right of the pose (f32 bound 1e-4 there)
    from exgame_b200 import _lib
    b = body(moments=(0.4, 0.4, 0.4))
    b["pose"] = _lib.motor_exp(np.array([10.0, 0, 0, 0, 0, 0]), 1.0)
    b["momentum"][3:] = [0.0, 0.0, 0.4]
    w = oracle.OracleWorld(np.array([b]), np.zeros(0, dtype=JOINT_DTYPE), step_params(integrator=LIE_EULER, dt=0.01))
    p0 = position(w.bodies()[0])
    w.step(100)
    p1 = position(w.bodies()[0])
    assert np.allclose(p0, [10.0, 0.0, 0.0], rtol=0, atol=1e-15)
    assert np.abs(p1 - p0).max() < 1e-12, (p0, p1)


def test_lie_free_linear_motion_is_uniform(oracle):
    # lie_euler.rs:162-180: mass 2, v = (3, 0, 0), 100 steps of 0.01: v stays 3 and x = v t = 3
    b = body(mass=2.0, vel=(3.0, 0.0, 0.0))
    w = oracle.OracleWorld(np.array([b]), np.zeros(0, dtype=JOINT_DTYPE), step_params(integrator=LIE_EULER, dt=0.01))
    w.step(100)
    bb = w.bodies()[0]
    assert np.allclose(bb["momentum"][:3] / 2.0, [3.0, 0.0, 0.0], rtol=0, atol=1e-13)
    assert np.allclose(position(bb), [3.0, 0.0, 0.0], rtol=0, atol=1e-12)


def test_euler_schemes_drift_more_than_lie(oracle):
    lie = world_momentum_drift(oracle, LIE_EULER, 0.01, 200)
    sym = world_momentum_drift(oracle, SYMPLECTIC_EULER, 0.01, 200)
    exp = world_momentum_drift(oracle, EXPLICIT_EULER, 0.01, 200)
    assert lie < 1e-9 < sym and lie < exp


# ── implicit Newton (crates/newton/src/integrator/implicit/newton.rs tests) ───────
def test_mass_block_is_diagonal_for_diagonal_inertia(oracle):
    # newton.rs:1041-1084
    b = body(mass=2.0, moments=(3.0, 5.0, 7.0))
    blk, rhs, sc = np.zeros(36), np.zeros(6), np.zeros(6)
    oracle.lib().orc_body_post(oracle.p(np.ascontiguousarray(b)), oracle.p(np.array([1.0, 0, 0, 0, 0, 0, 0, 0])),
                               oracle.p(np.zeros(6)), oracle.p(np.zeros(6)), oracle.p(np.zeros(6)), 0.5, 1e-18,
                               oracle.p(blk), oracle.p(rhs), oracle.p(sc))
    assert np.allclose(blk.reshape(6, 6), np.diag([2, 2, 2, 3, 5, 7]), atol=1e-12)


def test_newton_free_body_conserves_world_momentum_and_energy(oracle):
    # newton.rs:1093-1139 (bound 2e-2 in f32; the f64 restatement at tol 1e-10 does far better)
    b = body(moments=(2.0, 3.0, 4.0))
    b["momentum"][3:] = [2.0 * 1.0, 3.0 * 1.5, 4.0 * 0.7]
    w = oracle.OracleWorld(np.array([b]), np.zeros(0, dtype=JOINT_DTYPE), step_params(integrator=NEWTON, dt=0.01, tol=1e-10))
    from exgame_b200 import _lib
    l0 = _lib.screw_transport(b["momentum"], b["pose"], 1)[3:]
    e0 = w.energy()
    w.step(100)
    bb = w.bodies()[0]
    l1 = _lib.screw_transport(bb["momentum"], bb["pose"], 1)[3:]
    assert np.linalg.norm(l1 - l0) < 1e-6
    assert abs(w.energy() - e0) < 1e-4  # the reference bounds both by 2e-2


def test_newton_kinematic_body_does_not_stall_neighbour(oracle):
    # newton.rs:889-920
    bs = np.array([body((1, 0, 0)), body(kinematic=True)])
    w = oracle.OracleWorld(bs, np.array([spring(0, 1, 0.0, 10.0, 0.5)]), step_params(integrator=NEWTON, dt=1 / 60))
    x0 = position(w.bodies()[0])[0]
    w.step(200)
    x1 = position(w.bodies()[0])[0]
    assert np.isfinite(x1) and x1 < x0 - 0.05


def test_newton_stiff_nonlinear_step_matches_fine_lie_euler(oracle):
    # newton.rs:946-1027: k = 5e4, c = 5, rest 2, transverse speed 50, span 0.5 s, TOL 0.12
    def run(integrator, dt, steps):
        bs = np.array([body((1, 0, 0), (0, 50, 0)), body((-1, 0, 0), (0, -50, 0))])
        w = oracle.OracleWorld(bs, np.array([spring(0, 1, 2.0, 5e4, 5.0)]), step_params(integrator=integrator, dt=dt))
        w.step(steps)
        return np.array([position(b) for b in w.bodies()])
    ref = run(LIE_EULER, 1e-4, 5000)
    coarse = run(NEWTON, 0.002, 250)
    assert np.all(np.isfinite(coarse))
    assert np.abs(coarse - ref).max() < 0.12


def test_newton_equilibrium_is_held(oracle):
    # newton.rs:1337-1375: bodies at rest at the spring's rest length stay there
    bs = np.array([body((0, 0, 0)), body((2, 0, 0))])
    w = oracle.OracleWorld(bs, np.array([spring(0, 1, 2.0, 1e3, 1.0)]), step_params(integrator=NEWTON, dt=0.01, tol=1e-10))
    w.step(50)
    out = w.bodies()
    assert np.allclose(position(out[0]), [0, 0, 0], atol=1e-9)
    assert np.allclose(position(out[1]), [2, 0, 0], atol=1e-9)


def test_reference_newton_schulz_matches_exact_solve(oracle):
    # newton.rs:1140-1260: NS with a generous budget reproduces the exact solve (1e-6)
    bodies, joints = scenarios.chain_world(6, seed=11)
    p = step_params(integrator=NEWTON, dt=0.01, tol=1e-10)
    a = oracle.OracleWorld(bodies, joints, p, solver=oracle.OracleWorld.SOLVER_EXACT)
    b = oracle.OracleWorld(bodies, joints, p, solver=oracle.OracleWorld.SOLVER_REFERENCE_NS, ns_warm=8, ns_seed=40)
    a.step(20)
    b.step(20)
    pa = np.array([position(x) for x in a.bodies()])
    pb = np.array([position(x) for x in b.bodies()])
    assert np.abs(pa - pb).max() < 1e-6
    assert np.abs(a.bodies()["momentum"] - b.bodies()["momentum"]).max() < 1e-6


def test_reference_newton_schulz_default_budgets_converge(oracle):
    # the reference's own budgets (2 warm, 24 seed) reach the same step within the tolerance
    bodies, joints = scenarios.chain_world(6, seed=12)
    p = step_params(integrator=NEWTON, dt=0.01, tol=1e-8)
    a = oracle.OracleWorld(bodies, joints, p, solver=0)
    b = oracle.OracleWorld(bodies, joints, p, solver=1)
    a.step(10)
    b.step(10)
    pa = np.array([position(x) for x in a.bodies()])
    pb = np.array([position(x) for x in b.bodies()])
    assert np.abs(pa - pb).max() < 1e-5


def test_gravity_world_energy_drift_small(oracle):
    bodies = scenarios.gravity_world(64, 10.0, seed=3)
    w = oracle.OracleWorld(bodies, np.zeros(0, dtype=JOINT_DTYPE),
                           step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, softening=0.05, dt=1e-3))
    e0 = w.energy()
    w.step(200)
    assert abs(w.energy() - e0) / abs(e0) < 1e-3


def test_chain_generator_topology_bit_exact():
    """Joint topology and incidence order of the chain generator (the bit-exact part of parity)."""
    b, j = scenarios.chain_world(5, seed=1)
    assert list(j["law"]) == [0, 2, 3] * 4
    assert list(j["a"]) == [0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3]
    assert list(j["b"]) == [1, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 4]


def test_exact_pose_factor_converges_to_the_same_step(oracle):
    """The Newton matrix with the exact mid-point factor on the pose columns (-half^2/2) needs
    fewer iterations than the reference's (-half^2) and reaches the same step within tolerance."""
    bodies, joints = scenarios.chain_world(20, seed=17)
    ref = oracle.OracleWorld(bodies, joints, step_params(integrator=NEWTON, dt=1e-2, tol=1e-10))
    ex = oracle.OracleWorld(bodies, joints, step_params(integrator=NEWTON, dt=1e-2, tol=1e-10, exact_jacobian=True))
    its_ref, its_ex = 0, 0
    for _ in range(20):
        ref.step(1)
        ex.step(1)
        its_ref += ref.island_stats()[0][1]
        its_ex += ex.island_stats()[0][1]
    pa = np.array([position(x) for x in ref.bodies()])
    pb = np.array([position(x) for x in ex.bodies()])
    assert np.abs(pa - pb).max() < 1e-8
    assert its_ex < its_ref


def test_uniform_field_applies_m_times_accel_and_ignores_kinematic(oracle):
    """field.rs:54-97: with a world acceleration of gravity along -z plus a sideways +y wind, a
    dynamic body of mass 2 at the origin gets the world force m a; a kinematic body gets none.
    Restated through one LieEuler step: the momentum change is m a dt, the kinematic body is
    untouched."""
    from exgame_b200.abi import LIE_EULER, step_params
    m, a, dt = 2.0, (0.0, 1.5, -9.81), 0.01
    bs = np.array([body((0, 0, 0), (0, 0, 0), mass=m), body((3, 0, 0), kinematic=True)])
    w = oracle.OracleWorld(bs, np.zeros(0, dtype=JOINT_DTYPE), step_params(integrator=LIE_EULER, dt=dt, field=a))
    w.step(1)
    out = w.bodies()
    assert np.allclose(out[0]["momentum"][:3], np.array(a) * m * dt, rtol=0, atol=1e-15)
    assert np.array_equal(out[1]["momentum"], bs[1]["momentum"]) and np.array_equal(out[1]["pose"], bs[1]["pose"])
    # a free body in the field falls as p = 1/2 a t^2 under the implicit step too (tol 1e-10: the
    # body sits at its island's centre of mass, so its angular residual is measured against the
    # residual's floor, 1e-9, functions/src/lib.rs:170-247, which a tolerance of 1e-12 cannot meet)
    from exgame_b200.abi import NEWTON
    bs2 = np.array([body((1, 2, 3), (0, 0, 0), mass=m)])
    w2 = oracle.OracleWorld(bs2, np.zeros(0, dtype=JOINT_DTYPE),
                            step_params(integrator=NEWTON, dt=dt, tol=1e-10, field=a))
    w2.step(10)
    mom = w2.bodies()[0]["momentum"]
    assert np.allclose(mom[:3], np.array(a) * m * dt * 10, rtol=1e-9, atol=1e-12)


def test_bake_incidence_order_known_answer(oracle):
    """bake_incidence (crates/newton/src/accelerator/mod.rs:289-331): per body, the joint wrench
    slots in joint traversal order, end a (slot 0) before end b (slot 1); the cache's `order`
    enumerates the dynamic bodies in island order (integrator/implicit/cache.rs:566-573)."""
    from exgame_b200.abi import BODY_DTYPE, JOINT_DTYPE, NEWTON, step_params
    bodies = np.zeros(4, dtype=BODY_DTYPE)
    bodies["pose"][:, 0] = 1.0
    bodies["mass"] = 1.0
    bodies["inertia"][:, [0, 4, 8]] = 1.0
    bodies["diagonal"] = 1
    bodies["kinematic"][1] = 1
    joints = np.zeros(4, dtype=JOINT_DTYPE)
    for k, (a, b) in enumerate(((0, 1), (1, 2), (2, 0), (3, 2))):
        joints[k]["law"], joints[k]["a"], joints[k]["b"] = 3, a, b
        joints[k]["params"][0] = 1.0
    ow = oracle.OracleWorld(bodies, joints, step_params(integrator=NEWTON))
    assert ow.island_count() == 1
    assert list(ow.island_structure(0, "incidence_ptr")) == [0, 2, 4, 7, 8]
    # body 0: j0.a, j2.b; body 1: j0.b, j1.a; body 2: j1.b, j2.a, j3.b; body 3: j3.a
    assert list(ow.island_structure(0, "incidence")) == [0, 5, 1, 2, 3, 4, 7, 6]
    assert list(ow.island_structure(0, "order")) == [0, -1, 1, 2]
    assert ow.island_structure(0, "joint_ends").tolist() == [[3, 0, 1], [3, 1, 2], [3, 2, 0], [3, 3, 2]]
