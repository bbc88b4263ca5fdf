"""The C ABI: the library loads without a GPU, exports every symbol include/exg.h declares, and
its record layouts match the oracle's view of the same header."""
import os
import re
import subprocess

import numpy as np
import pytest

from exgame_b200 import _lib
from exgame_b200.abi import BODY_DTYPE, JOINT_DTYPE, LAW_N_PARAMS, LAW_NAMES, STEP_PARAMS_DTYPE, WORLD_STATS_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "exg.h")).read()
    return sorted(set(re.findall(r"EXG_API\s+[\w\s\*]+?\b(exg_\w+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ("exg_device_create", "exg_world_create", "exg_world_step", "exg_eval_joints", "exg_gravity_forces"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (exg_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    assert set(declared_symbols()) == set(_lib.SIGNATURES), "ctypes table out of sync with the header"


def test_library_loads_without_device_and_binds():
    L = _lib.lib()
    assert L.exg_abi_version() == 1
    assert L.exg_status_string(-1).decode() == "no kernel for this joint law"


def test_record_layouts_match_c(oracle):
    L = oracle.lib()
    assert BODY_DTYPE.itemsize == L.orc_body_size() == 208
    assert JOINT_DTYPE.itemsize == L.orc_joint_size() == 96
    assert STEP_PARAMS_DTYPE.itemsize == 64
    assert WORLD_STATS_DTYPE.itemsize == 32


def test_law_lookup_by_shader_name():
    # crates/newton/src/accelerator/mod.rs:118-132
    for k, name in enumerate(LAW_NAMES):
        assert _lib.law_lookup(name) == (k, LAW_N_PARAMS[k])
    with pytest.raises(_lib.ExgError) as e:
        _lib.law_lookup("NoSuchLaw")
    assert e.value.name == "EXG_ERR_NO_SHADER"


def test_device_create_reports_no_device_cleanly():
    import ctypes
    h = ctypes.c_void_p()
    st = _lib.lib().exg_device_create(10_000, ctypes.byref(h))
    assert st in (-24, -20)  # no device here, or an out-of-range ordinal on a GPU box


def test_host_motor_utilities_match_oracle(oracle):
    rng = np.random.default_rng(5)
    for _ in range(10):
        t = rng.normal(size=6)
        m = _lib.motor_exp(t, 0.7)
        assert np.array_equal(m, oracle.twist_exp(t, 0.7))
        q = rng.normal(size=3)
        assert np.allclose(_lib.motor_apply_point(m, q), _lib.motor_apply_point(m, q))
    # rotation by +90 degrees about z moves (1,0,0) to (0,1,0) (crates/clifford/src/pga3/motor.rs:343-352)
    m = _lib.motor_exp([0, 0, 0, 0, 0, np.pi / 2], 1.0)
    assert np.allclose(_lib.motor_apply_point(m, [1, 0, 0]), [0, 1, 0], atol=1e-12)
    # translation by (2,0,0) moves the origin to (2,0,0) (motor.rs:354-363)
    m = _lib.motor_exp([2, 0, 0, 0, 0, 0], 1.0)
    assert np.allclose(_lib.motor_apply_point(m, [0, 0, 0]), [2, 0, 0], atol=1e-12)
    # compose is "first a, then b": translate then rotate about the origin
    a = _lib.motor_exp([1, 0, 0, 0, 0, 0], 1.0)
    b = _lib.motor_exp([0, 0, 0, 0, 0, np.pi / 2], 1.0)
    assert np.allclose(_lib.motor_apply_point(_lib.motor_compose(a, b), [0, 0, 0]), [0, 1, 0], atol=1e-12)
