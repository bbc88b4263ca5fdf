"""The device algebra and force-law headers of the CUDA path, compiled for the host, against the
oracle: slot order, signs and the Jacobian slices are checked here without a GPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "devalg_host.cpp")
OUT = os.path.join(HERE, "native", "_build", "libdevalg_host.so")


@pytest.fixture(scope="module")
def dh():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", OUT, SRC], check=True)
    L = ctypes.CDLL(OUT)
    L.dh_power.restype = ctypes.c_double
    for fn in ("dh_joint_plain", "dh_joint_jacobian"):
        getattr(L, fn).argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 5 + [ctypes.c_double, ctypes.c_double,
                                                                               ctypes.c_void_p]
    L.dh_twist_exp.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    return L


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_motor_algebra_matches_oracle(dh, oracle):
    rng = np.random.default_rng(0)
    for _ in range(25):
        t1, t2 = rng.normal(size=6), rng.normal(size=6)
        m_d = np.zeros(8)
        dh.dh_twist_exp(P(t1), 0.8, P(m_d))
        m_o = oracle.twist_exp(t1, 0.8)
        assert np.allclose(m_d, m_o, rtol=0, atol=1e-15)
        for co in (0, 1):
            a, b = np.zeros(6), np.zeros(6)
            dh.dh_transport(P(t2), P(m_o), co, P(a))
            oracle.lib().orc_twist_transport(oracle.p(t2), oracle.p(m_o), co, oracle.p(b))
            assert np.allclose(a, b, atol=1e-14)
        r_d, r_o = np.zeros(6), np.zeros(6)
        dh.dh_coad(P(t1), P(t2), P(r_d))
        oracle.lib().orc_coad_bracket(oracle.p(t1), oracle.p(t2), oracle.p(r_o))
        assert np.allclose(r_d, r_o, atol=1e-14)


@pytest.mark.parametrize("law", [0, 1, 2, 3])
def test_joint_plain_and_jacobian_match_oracle(dh, oracle, law):
    rng = np.random.default_rng(10 + law)
    for _ in range(10):
        prm = np.zeros(10)
        prm[:6] = rng.normal(size=6) * 0.3
        prm[6:10] = [1.3, 7.0, 2.0, 1e-6]
        if law == 2:
            prm[:2] = [2.0, 1e-3]
        if law == 3:
            prm[0] = 1.5
        pa, pb = oracle.twist_exp(rng.normal(size=6)), oracle.twist_exp(rng.normal(size=6))
        va, vb = rng.normal(size=6), rng.normal(size=6)
        out = np.zeros(12)
        dh.dh_joint_plain(law, P(prm), P(pa), P(pb), P(va), P(vb), 0.016, 1.3, P(out))
        want = oracle.plain_eval(law, prm, pa, pb, va, vb, 0.016, 1.3)
        assert np.allclose(out, want, rtol=1e-13, atol=1e-13)
        jac = np.zeros(300)
        dh.dh_joint_jacobian(law, P(prm), P(pa), P(pb), P(va), P(vb), 0.016, 1.3, P(jac))
        wj = oracle.jacobian_eval(law, prm, pa, pb, va, vb, 0.016, 1.3)
        assert np.allclose(jac.reshape(12, 25), wj, rtol=1e-12, atol=1e-12)
        assert np.array_equal(jac.reshape(12, 25)[:, 0], out)  # Jacobian kernel value == plain value


def test_half_slices_equal_whole_slices_bit_for_bit(dh):
    """A Jacobian slice evaluated as two 3-axis halves (what the wave's joint kernels do) equals the
    6-axis slice bit for bit, in FP64 and FP32, for every law."""
    rng = np.random.default_rng(12)
    from exgame_b200 import _lib
    for law in range(4):
        for _ in range(5):
            prm = rng.normal(size=10)
            prm[6:9] = np.abs(prm[6:9]) + 0.5
            prm[9] = 1e-6
            if law >= 2:
                prm[:2] = np.abs(prm[:2])
            pa = _lib.motor_exp(rng.normal(size=6), 1.0)
            pb = _lib.motor_exp(rng.normal(size=6), 1.0)
            va, vb = rng.normal(size=6), rng.normal(size=6)
            whole, halves = np.zeros(300), np.zeros(300)
            args = (law, P(prm), P(pa), P(pb), P(va), P(vb), ctypes.c_double(0.016), ctypes.c_double(1.3))
            dh.dh_joint_jacobian(*args, P(whole))
            dh.dh_joint_jacobian_halves.argtypes = dh.dh_joint_jacobian.argtypes
            dh.dh_joint_jacobian_halves(*args, P(halves))
            assert np.array_equal(whole, halves), law
            f = [np.ascontiguousarray(x, dtype=np.float32) for x in (pa, pb, va, vb)]
            o6, o3 = np.zeros(168, np.float32), np.zeros(168, np.float32)
            dh.dh_jacobian_slices_f32(law, P(prm), *[P(x) for x in f], ctypes.c_double(0.016), ctypes.c_double(1.3), 0,
                                      P(o6))
            dh.dh_jacobian_slices_f32(law, P(prm), *[P(x) for x in f], ctypes.c_double(0.016), ctypes.c_double(1.3), 1,
                                      P(o3))
            assert np.array_equal(o6, o3), law


# ── the device's dual-number carrier (exg::Dual, csrc/scalar.cuh) against the reference's
# first-order Tangent tests (crates/clifford/src/tangent.rs:340-510) ──

ADD, SUB, MUL, DIV, RECIP, SQRT, SIN, COS, ATAN2, EXP, LOG, ABS, FOO, SIN_SQ, EXP_LOG = range(15)


def dual(dh, op, a, da=1.0, b=0.0, db=0.0):
    out = np.zeros(2)
    dh.dh_dual1.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [ctypes.c_void_p]
    dh.dh_dual1(op, a, da, b, db, P(out))
    return out


def test_dual_simple_and_product_rules(dh):
    # tangent.rs:383-391 `simple`: a = (10, 2), b = (2, 2), a b + a / b = (25, 20)
    assert list(dual(dh, FOO, 10.0, 2.0, 2.0, 2.0)) == [25.0, 20.0]
    # tangent.rs:421-439: constant, x^2 at 3 -> (9, 6), 1/x at 2 -> (0.5, -0.25)
    assert list(dual(dh, MUL, 7.0, 0.0, 3.0, 0.0)) == [21.0, 0.0]
    assert list(dual(dh, MUL, 3.0, 1.0, 3.0, 1.0)) == [9.0, 6.0]
    assert list(dual(dh, RECIP, 2.0)) == [0.5, -0.25]
    assert list(dual(dh, DIV, 1.0, 0.0, 2.0, 1.0)) == [0.5, -0.25]


def test_dual_transcendentals(dh):
    # tangent.rs:441-470: sqrt at 4 -> (2, 1/4); exp(ln x) at 3 -> (3, 1); sin, cos at 0; sin(x^2) at 1
    v, d = dual(dh, SQRT, 4.0)
    assert abs(v - 2.0) < 1e-12 and abs(d - 0.25) < 1e-12
    v, d = dual(dh, EXP_LOG, 3.0)
    assert abs(v - 3.0) < 1e-12 and abs(d - 1.0) < 1e-12
    assert np.allclose(dual(dh, SIN, 0.0), [0.0, 1.0], rtol=0, atol=1e-15)
    assert np.allclose(dual(dh, COS, 0.0), [1.0, 0.0], rtol=0, atol=1e-15)
    v, d = dual(dh, SIN_SQ, 1.0)
    assert abs(v - np.sin(1.0)) < 1e-12 and abs(d - 2.0 * np.cos(1.0)) < 1e-12
    v, d = dual(dh, EXP, 0.5)
    assert abs(v - np.exp(0.5)) < 1e-12 and abs(d - np.exp(0.5)) < 1e-12
    v, d = dual(dh, LOG, 2.0)
    assert abs(v - np.log(2.0)) < 1e-12 and abs(d - 0.5) < 1e-12


def test_dual_atan2(dh):
    # tangent.rs:490-505: atan2(sin t, cos t) at t = 0.7 -> (0.7, 1); d/dy atan2(y, x) at (1, 2) = x / (x^2 + y^2)
    t = 0.7
    s, ds = dual(dh, SIN, t)
    c, dc = dual(dh, COS, t)
    v, d = dual(dh, ATAN2, s, ds, c, dc)
    assert abs(v - 0.7) < 1e-12 and abs(d - 1.0) < 1e-12
    v, d = dual(dh, ATAN2, 1.0, 1.0, 2.0, 0.0)
    assert abs(v - np.arctan2(1.0, 2.0)) < 1e-15 and abs(d - 2.0 / 5.0) < 1e-15
    # and the x partial: -y / (x^2 + y^2)
    v, d = dual(dh, ATAN2, 1.0, 0.0, 2.0, 1.0)
    assert abs(d + 1.0 / 5.0) < 1e-15


def test_dual_singular_points_stay_finite_in_value(dh):
    # tangent.rs:347-360: sqrt and ln at 0 must not abort; the value of sqrt is clean, only the
    # derivative is non-finite (a downstream guard on the standard part discards it)
    v, d = dual(dh, SQRT, 0.0)
    assert v == 0.0 and not np.isfinite(d)
    v, d = dual(dh, LOG, 0.0)
    assert v == -np.inf
    # |x| takes derivative sign(x), 0 at 0
    assert list(dual(dh, ABS, -2.0)) == [2.0, -1.0] and list(dual(dh, ABS, 0.0)) == [0.0, 0.0]


def test_study_forms_match_the_oracle_across_the_seams(dh, oracle):
    """The device's Study forms (the exp of a twist goes through them) against the oracle's
    restatement of crates/peano/src/scalar.rs:67-131 with the thresholds of support.rs:39-49,
    on both sides of every seam (f64: |u| < 1e-9, and 1e-4 for the derivative's arm; f32: 1e-5
    and 1), bit for bit: the same arms, the same operation order."""
    dh.dh_study_forms.argtypes = [ctypes.c_double, ctypes.c_void_p]
    dh.dh_study_forms_f32.argtypes = [ctypes.c_float, ctypes.c_void_p]
    L = oracle.lib()
    us = np.r_[0.0, np.logspace(-14, 1.5, 400), 0.999e-9, 1.001e-9, 0.999e-4, 1.001e-4, 0.999e-5, 1.001e-5, 0.999,
               1.001]
    for u in us:
        d, o = np.zeros(3), np.zeros(3)
        dh.dh_study_forms(float(u), P(d))
        L.orc_study_forms(ctypes.c_double(u), oracle.p(o))
        assert np.array_equal(d, o), (u, d, o)
        df, of = np.zeros(3, dtype=np.float32), np.zeros(3, dtype=np.float32)
        dh.dh_study_forms_f32(np.float32(u), P(df))
        L.orc_study_forms_f32(ctypes.c_float(u), ctypes.c_void_p(of.ctypes.data))
        assert np.array_equal(df, of), (u, df, of)


def test_inertia_and_world_velocity_match_the_oracle(dh, oracle):
    """The device's inertia apply / inverse (crates/newton/src/inertia.rs:271-345) for diagonal,
    full-tensor and kinematic bodies, and its world twist of a body (Ad_pose of I^-1 P,
    crates/newton/src/body.rs:141-186) against numpy's solve and the oracle's transport."""
    dh.dh_inertia.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                              ctypes.c_void_p, ctypes.c_void_p]
    dh.dh_world_velocity.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                             ctypes.c_void_p]
    rng = np.random.default_rng(5)
    for case in range(60):
        kin = case % 5 == 4
        diag = case % 2 == 0
        mass = 0.0 if kin else float(rng.uniform(0.2, 5.0))
        if diag:
            I = np.diag(rng.uniform(0.2, 4.0, size=3))
        else:
            A = rng.normal(size=(3, 3))
            I = A @ A.T + 0.5 * np.eye(3)
        I9 = np.ascontiguousarray(I.reshape(-1))
        p6 = rng.normal(size=6)
        v6, back = np.zeros(6), np.zeros(6)
        dh.dh_inertia(P(I9), int(diag), int(kin), mass, 1, P(p6), P(v6))
        want = p6.copy() if kin else np.r_[p6[:3] / mass, np.linalg.solve(I, p6[3:])]
        assert np.allclose(v6, want, rtol=1e-13, atol=1e-13), case
        dh.dh_inertia(P(I9), int(diag), int(kin), mass, 0, P(v6), P(back))
        assert np.allclose(back, p6, rtol=1e-12, atol=1e-12), case
        pose = oracle.twist_exp(rng.normal(size=6))
        wv, ref = np.zeros(6), np.zeros(6)
        dh.dh_world_velocity(P(pose), P(p6), P(I9), int(diag), int(kin), mass, P(wv))
        oracle.lib().orc_twist_transport(oracle.p(oracle.arr(want)), oracle.p(pose), 0, oracle.p(ref))
        assert np.allclose(wv, ref, rtol=1e-12, atol=1e-12), case
