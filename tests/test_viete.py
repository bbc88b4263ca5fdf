"""viete, the tracer and CUDA C emitter of joint force laws (crates/viete/src/api.rs, ir.rs,
glsl.rs; the reference emits GLSL, this package emits CUDA C). The traced laws of
exgame_b200/user_laws.py are compiled for the host from the generated header together with the
device algebra and checked: the traced restatement of SimpleSpringDamper against the oracle's law
(plain values and the 24-axis Jacobian), the new PointBushing against its own float evaluation and
against finite differences of it, and the law registry of the C ABI."""
import ctypes
import math
import os
import subprocess

import numpy as np
import pytest

from exgame_b200 import _lib, motors_np, pga_sym, user_laws, viete

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "devalg_host.cpp")
OUT = os.path.join(HERE, "native", "_build", "libdevalg_viete.so")


@pytest.fixture(scope="module")
def dh():
    viete.generate()
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", OUT, SRC], check=True)
    L = ctypes.CDLL(OUT)
    for fn in ("dh_joint_plain", "dh_joint_jacobian"):
        getattr(L, fn).argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 5 + [ctypes.c_double, ctypes.c_double,
                                                                               ctypes.c_void_p]
    return L


def P(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.c_void_p)


def case(rng):
    pa = motors_np.twist_exp_n(rng.normal(size=6) * 0.7, 1.0)[0]
    pb = motors_np.twist_exp_n(rng.normal(size=6) * 0.7 + np.array([2.0, 0.5, 0, 0, 0, 0]), 1.0)[0]
    return pa, pb, rng.normal(size=6), rng.normal(size=6)


def host_plain(dh, law, prm, pa, pb, va, vb, dt=0.016, warp=1.3):
    out = np.zeros(12)
    prm = np.ascontiguousarray(prm, dtype=np.float64)
    dh.dh_joint_plain(law, P(prm), P(pa), P(pb), P(va), P(vb), dt, warp, out.ctypes.data_as(ctypes.c_void_p))
    return out


def host_jacobian(dh, law, prm, pa, pb, va, vb, dt=0.016, warp=1.3):
    out = np.zeros(300)
    prm = np.ascontiguousarray(prm, dtype=np.float64)
    dh.dh_joint_jacobian(law, P(prm), P(pa), P(pb), P(va), P(vb), dt, warp, out.ctypes.data_as(ctypes.c_void_p))
    return out.reshape(12, 25)


def spring_params(rng):
    prm = np.zeros(10)
    prm[0:6] = rng.normal(size=6) * 0.3
    prm[6:10] = (1.3, 7.0, 2.0, 1e-6)
    return prm


def test_traced_spring_damper_equals_the_oracle_law(dh, oracle):
    """The traced restatement (law 4) against the oracle's SimpleSpringDamper (law 0)."""
    rng = np.random.default_rng(11)
    for _ in range(30):
        prm = spring_params(rng)
        pa, pb, va, vb = case(rng)
        got = host_plain(dh, 4, prm, pa, pb, va, vb)
        want = oracle.plain_eval(0, prm, pa, pb, va, vb, 0.016, 1.3)
        assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()
        gj = host_jacobian(dh, 4, prm, pa, pb, va, vb)
        wj = oracle.jacobian_eval(0, prm, pa, pb, va, vb, 0.016, 1.3)
        assert np.abs(gj - wj).max() <= 1e-12 * np.abs(wj).max()


def bushing_float(prm, pa, pb, va, vb, warp=1.3):
    """PointBushing evaluated with floats through the same Python definition the tracer ran."""
    class Ctx:
        pass
    c = Ctx()
    c.params = list(map(float, prm))
    c.pose_a, c.pose_b = pga_sym.motor(list(pa)), pga_sym.motor(list(pb))
    c.twist_a = pga_sym.screw(list(va[:3]), list(va[3:]))
    c.twist_b = pga_sym.screw(list(vb[:3]), list(vb[3:]))
    c.dt, c.warp = 0.016, warp
    w = user_laws.point_bushing(c)
    lin, ang = pga_sym.screw_parts(w)
    return np.array(lin + ang)


def test_point_bushing_emitted_code_matches_its_definition(dh):
    rng = np.random.default_rng(12)
    for _ in range(30):
        prm = np.concatenate([rng.normal(size=6) * 0.3, [50.0, 3.0]])
        pa, pb, va, vb = case(rng)
        got = host_plain(dh, 5, prm, pa, pb, va, vb)
        want = bushing_float(prm, pa, pb, va, vb)
        assert np.abs(got[:6] - want).max() <= 1e-13 * np.abs(want).max()
        assert np.array_equal(got[6:], -got[:6])


def test_point_bushing_jacobian_matches_finite_differences(dh):
    """The dual evaluation of the emitted law against central differences of its definition along
    the 24 axes: pose A, pose B (retraction exp(delta) * pose), twist A, twist B."""
    rng = np.random.default_rng(13)
    h = 1e-6
    for _ in range(5):
        prm = np.concatenate([rng.normal(size=6) * 0.3, [50.0, 3.0]])
        pa, pb, va, vb = case(rng)
        J = host_jacobian(dh, 5, prm, pa, pb, va, vb)
        for axis in range(24):
            d = np.zeros(6)
            d[axis % 6] = h
            args_p, args_m = [pa, pb, va, vb], [pa, pb, va, vb]
            k = axis // 6
            if k < 2:  # Motor::exp(delta) * pose (unit exp: Twist::exp(2 delta) halves it back)
                base = (pa, pb)[k]
                args_p[k] = motors_np.compose_n(base, motors_np.twist_exp_n(2 * d, 1.0))[0]
                args_m[k] = motors_np.compose_n(base, motors_np.twist_exp_n(-2 * d, 1.0))[0]
            else:
                args_p[k] = (va, vb)[k - 2] + d
                args_m[k] = (va, vb)[k - 2] - d
            fd = (bushing_float(prm, *args_p) - bushing_float(prm, *args_m)) / (2 * h)
            scale = max(1.0, np.abs(J[:6, 1:]).max())
            assert np.abs(J[:6, 1 + axis] - fd).max() <= 2e-6 * scale, axis


def test_trace_records_live_ops_only_and_refuses_branches():
    law = viete.TracedLaw("TracedSpringDamper", 10, user_laws.traced_spring_damper)
    counts = law.counts()
    assert counts["sqrt"] == 1 and counts["div"] == 1 and "in" not in counts
    text = viete.emit_cuda(law, 0)
    assert "template <class S, class P = S>" in text and "Lift<S>::from(" in text
    tr = viete.Trace()
    x = tr.new(2, "in", ("ta", 0))
    with pytest.raises(TypeError):
        if x < 1.0:
            pass
    assert viete.sqrt(4.0) == 2.0 and viete.atan2(1.0, 1.0) == math.atan2(1.0, 1.0)


def test_law_registry_finds_the_traced_laws():
    for k, (name, n, _) in enumerate(user_laws.LAWS):
        law, n_params = _lib.law_lookup(name)
        assert law == 4 + k and n_params == n
    with pytest.raises(_lib.ExgError):
        _lib.law_lookup("NoSuchLaw")
