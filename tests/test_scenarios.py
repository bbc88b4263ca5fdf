"""The workload generator's numpy motor algebra against the oracle, and the generator's
independence from the CUDA library (the CPU baseline builds its inputs without it)."""
import subprocess
import sys

import numpy as np

from exgame_b200 import motors_np, scenarios


def test_twist_exp_and_compose_match_the_oracle_bit_for_bit(oracle):
    rng = np.random.default_rng(7)
    t = rng.normal(size=(300, 6)) * np.array([3.0, 3.0, 3.0, 1.0, 1.0, 1.0])
    t[:40] *= 1e-6   # the Taylor arms of the Study forms (|u| < 1e-9 and |u 1e-5| < 1e-9)
    t[40:60] *= 1e-3
    got = motors_np.twist_exp_n(t, 0.7)
    want = np.array([oracle.twist_exp(x, 0.7) for x in t])
    assert np.array_equal(got, want)
    L = oracle.lib()
    a, b = got[:150], got[150:]
    comp = motors_np.compose_n(a, b)
    for k in range(150):
        o = np.zeros(8)
        L.orc_motor_compose(oracle.p(oracle.arr(a[k])), oracle.p(oracle.arr(b[k])), oracle.p(o))
        assert np.array_equal(comp[k], o)


def test_apply_point_matches_the_oracle(oracle):
    rng = np.random.default_rng(8)
    m = motors_np.twist_exp_n(rng.normal(size=(100, 6)), 1.0)
    p = rng.normal(size=(100, 3))
    got = motors_np.apply_point_n(m, p)
    L = oracle.lib()
    for k in range(100):
        o = np.zeros(3)
        L.orc_motor_apply_point(oracle.p(oracle.arr(m[k])), oracle.p(oracle.arr(p[k])), oracle.p(o))
        assert np.abs(got[k] - o).max() <= 1e-14 * max(1.0, np.abs(o).max())


def test_generated_poses_are_unit_motors():
    b, _ = scenarios.tree_world(200, seed=3)
    m = b["pose"]
    # a motor's norm: scalar^2 + the Euclidean bivector's squares = 1; the pseudoscalar weight
    # pairs with the scalar against the radical part (m m~ has no pseudoscalar)
    assert np.allclose(m[:, 0] ** 2 + m[:, 1] ** 2 + m[:, 2] ** 2 + m[:, 3] ** 2, 1.0, atol=1e-14)


def test_generating_workloads_loads_no_cuda_library():
    code = ("import sys; from exgame_b200 import scenarios, _lib; scenarios.config3_worlds(16); "
            "scenarios.config2_parts(n_gravity=64, n_chains=2, chain_len=8); "
            "assert _lib._LIB is None, 'libexg loaded'; print('ok')")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=scenarios.__file__.rsplit(
        "/exgame_b200/", 1)[0])
    assert out.returncode == 0 and "ok" in out.stdout, out.stderr
