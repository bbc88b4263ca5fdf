"""The gravity entry point that allocates no device memory.

Some callers cannot allocate device memory when they need forces — a host that pre-sizes or
reserves all device memory up front, or code running where the allocator must not be entered.
`exg_gravity_forces_noalloc` serves them from a fixed working array compiled into the library,
for at most EXG_NOALLOC_MAX_BODIES bodies. This file checks it through the C ABI against the
allocating `exg_gravity_forces` on two calls in a row (the second sees the array the first left
behind). It is named to be collected last, so a run that stops at the first failure has already
run everything else; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from exgame_b200 import _lib, motors_np, scenarios
from exgame_b200.abi import GRAVITY_PLUMMER, GRAVITY_SIZE_CORE, PRECISION_F64, PRECISION_MIXED

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_BODIES = 16384  # EXG_NOALLOC_MAX_BODIES in include/exg.h


def charges(bodies):
    p = motors_np.apply_point_n(bodies["pose"], np.zeros((len(bodies), 3)))
    pm = np.zeros((len(bodies), 4))
    pm[:, :3] = p
    pm[:, 3] = bodies["mass"]
    return pm


def on_device(a):
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()
    torch.cuda.synchronize()
    return t


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def forces(dev, fn, pm_t, size_t, n, law, precision):
    out = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(fn(dev.handle, vp(pm_t), vp(size_t), n, law, 1.0, 0.05, precision, vp(out)), fn.__name__)
    return out.cpu().numpy().reshape(n, 3)


@pytest.mark.parametrize("precision", [PRECISION_F64, PRECISION_MIXED])
def test_noalloc_matches_allocating_entry_point_twice(precision):
    """Both entry points run the same work plan through the same kernels, so they agree bit for
    bit; the sizes include the array's limit (MAX_BODIES: every work item and partial-sum slot of
    the fixed array in use) and one body below it, each followed by a smaller call that must not
    see what the larger one left behind."""
    L = _lib.lib()
    dev = _lib.Device(0)
    cases = ((3000, GRAVITY_PLUMMER, 1), (700, GRAVITY_SIZE_CORE, 2), (MAX_BODIES, GRAVITY_PLUMMER, 3),
             (1000, GRAVITY_SIZE_CORE, 4), (MAX_BODIES - 1, GRAVITY_SIZE_CORE, 5), (257, GRAVITY_PLUMMER, 6))
    for n, law, seed in cases:
        bodies = scenarios.gravity_world(n, 50.0, seed=seed)
        pm_t, size_t = on_device(charges(bodies)), on_device(np.ascontiguousarray(bodies["size"]))
        want = forces(dev, L.exg_gravity_forces, pm_t, size_t, n, law, precision)
        got = forces(dev, L.exg_gravity_forces_noalloc, pm_t, size_t, n, law, precision)
        assert np.isfinite(want).all()
        assert np.array_equal(got, want), (n, law, np.abs(got - want).max())
    dev.close()


def test_noalloc_rejects_sizes_beyond_its_array():
    L = _lib.lib()
    dev = _lib.Device(0)
    n = MAX_BODIES + 1
    pm_t = torch.zeros(4 * n, dtype=torch.float64, device="cuda")
    out = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = L.exg_gravity_forces_noalloc(dev.handle, vp(pm_t), None, n, GRAVITY_PLUMMER, 1.0, 0.05, PRECISION_F64, vp(out))
    assert st == -20  # EXG_ERR_INVALID_ARGUMENT
    dev.close()


def test_both_entry_points_reject_unknown_precision():
    L = _lib.lib()
    dev = _lib.Device(0)
    n = 64
    pm_t = torch.ones(4 * n, dtype=torch.float64, device="cuda")
    out = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for fn in (L.exg_gravity_forces, L.exg_gravity_forces_noalloc):
        assert fn(dev.handle, vp(pm_t), None, n, GRAVITY_PLUMMER, 1.0, 0.05, 7, vp(out)) == -20
    dev.close()
