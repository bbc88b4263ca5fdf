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
    assert L.exg_abi_version() == 2
    assert L.exg_status_string(-1).decode() == "no kernel for this joint law"


def test_record_layouts_match_c(oracle):
    L = oracle.lib()
    assert BODY_DTYPE.itemsize == L.orc_body_size() == 208
    assert JOINT_DTYPE.itemsize == L.orc_joint_size() == 96
    assert STEP_PARAMS_DTYPE.itemsize == 88
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


def test_every_record_dtype_matches_the_compiled_header(tmp_path):
    """Compile a layout probe against include/exg.h with the host C compiler and compare each
    record's size and field offsets with the numpy dtype the binding passes by pointer."""
    from exgame_b200 import abi
    exe = tmp_path / "abi_layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", str(exe),
                    os.path.join(ROOT, "tests", "native", "abi_layout.c")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    dtypes = {"exg_body_t": abi.BODY_DTYPE, "exg_joint_t": abi.JOINT_DTYPE, "exg_step_params_t": abi.STEP_PARAMS_DTYPE,
              "exg_world_stats_t": abi.WORLD_STATS_DTYPE, "exg_pool_config_t": abi.POOL_CONFIG_DTYPE,
              "exg_pool_usage_t": abi.POOL_USAGE_DTYPE, "exg_server_config_t": abi.SERVER_CONFIG_DTYPE,
              "exg_request_info_t": abi.REQUEST_INFO_DTYPE, "exg_server_stats_t": abi.SERVER_STATS_DTYPE}
    checked = 0
    for line in out:
        if not line:
            continue
        t, field, value = line.split()
        dt = dtypes[t]
        if field == "sizeof":
            assert dt.itemsize == int(value), t
        else:
            assert dt.fields[field][1] == int(value), (t, field)
        checked += 1
    assert checked > 60


def test_world_footprint_without_device():
    from exgame_b200 import abi
    from exgame_b200._lib import world_footprint
    free = world_footprint(1000, 0, abi.step_params())
    grav = world_footprint(1000, 0, abi.step_params(gravity_law=abi.GRAVITY_PLUMMER, softening=0.05))
    newton = world_footprint(1000, 999, abi.step_params(integrator=abi.NEWTON))
    assert 0 < free < grav < newton
    assert world_footprint(2000, 0, abi.step_params()) == 2 * free
    with pytest.raises(_lib.ExgError):
        world_footprint(-1, 0, abi.step_params())


def test_pool_and_server_reject_a_missing_device():
    import ctypes
    from exgame_b200 import abi
    cfg = np.zeros((), dtype=abi.SERVER_CONFIG_DTYPE)
    cfg["hbm_budget_bytes"], cfg["max_bodies"], cfg["max_worlds"], cfg["steps_per_tick"] = 1 << 30, 1024, 4, 8
    h = ctypes.c_void_p()
    assert _lib.lib().exg_server_create(None, _lib.ptr(cfg), ctypes.byref(h)) == -20
    pc = np.zeros((), dtype=abi.POOL_CONFIG_DTYPE)
    pc["max_bodies"], pc["max_worlds"] = 1024, 4
    assert _lib.lib().exg_pool_create(None, _lib.ptr(pc), ctypes.byref(h)) == -20


def test_ledger_refuses_a_second_writer_and_out_of_range_slots():
    """The one-writer check (crates/newton/src/accelerator/shaders.rs:321-390) is host only."""
    assert _lib.ledger_check([3, 1, 4, 0, 2], 5) == (0, -1)
    st, at = _lib.ledger_check([3, 1, 4, 1, 2], 5)
    assert st == -5 and at == 3
    assert "second writer" in _lib.lib().exg_status_string(st).decode()
    st, at = _lib.ledger_check([0, 7], 5)
    assert st == -5 and at == 1
    assert _lib.ledger_check([], 0) == (0, -1)
