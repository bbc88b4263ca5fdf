"""The implicit solve's 6x6 pivot inverse through the C ABI (exg_pivot_inverse).

The mixed path inverts each pivot block by FP32 Newton-Schulz iterations on the diagonally scaled
block, seeded with the identity where that block is close to it, else with the reference's
transposed seed (seed_transpose, crates/newton/src/integrator/implicit/newton.rs:209-241), then
one FP64 Newton-Schulz correction; the plain path by FP64 Gauss-Jordan. Checked here:
  - the thread form (wide elimination levels) and the warp form (narrow levels, island kernel)
    give the same bits, for both methods, so the two Newton schedules stay bit-identical;
  - the mixed inverse's error against the FP64 inverse: max |D X - I| <= 1e-11 on pivot-like
    blocks (mass block of a box + dt^2 stiffness + dt damping and gyroscopic terms), and its FP32
    step count (a median of at most 6 on them);
  - a block too ill-conditioned for FP32 falls back to Gauss-Jordan (steps -1) and still inverts;
  - a singular block is reported (EXG_ERR_FATAL).
"""
import ctypes

import numpy as np
import pytest

from exgame_b200 import _lib
from exgame_b200.abi import PRECISION_F64, PRECISION_MIXED

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def pivot_like_blocks(n, seed):
    """Blocks of the kind the elimination inverts: a rigid body's mass block (mass 8 hx hy hz of a
    box with half-extents in [0.5, 2], density 1, and its rotated inertia tensor) plus dt^2 times
    a stiffness block of joint springs (k log-uniform in [1e2, 1e4]) and dt times damping and a
    gyroscopic skew term, dt = 1e-2."""
    rng = np.random.default_rng(seed)
    dt = 1e-2
    out = np.zeros((n, 6, 6))
    for b in range(n):
        h = rng.uniform(0.5, 2.0, 3)
        m = 8.0 * h.prod()
        ib = m / 3.0 * np.array([h[1] ** 2 + h[2] ** 2, h[0] ** 2 + h[2] ** 2, h[0] ** 2 + h[1] ** 2])
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        M = np.zeros((6, 6))
        M[:3, :3] = m * np.eye(3)
        M[3:, 3:] = q @ np.diag(ib) @ q.T
        K = np.zeros((6, 6))
        for _ in range(int(rng.integers(1, 4))):  # a few incident springs
            J = rng.normal(size=(3, 6))
            K += 10.0 ** rng.uniform(2, 4) * (J.T @ J)
        C = 0.1 * np.sqrt(1e3) * np.diag(rng.uniform(0, 1, 6))
        w = rng.normal(size=3)
        G = np.zeros((6, 6))
        G[3:, 3:] = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]]) @ M[3:, 3:]
        out[b] = M + dt * dt * K + dt * (C + G)
    return out


def run(device, blocks, precision, form, prev=None):
    n = len(blocks)
    d_in = torch.from_numpy(np.ascontiguousarray(blocks).reshape(-1).copy()).cuda()
    if prev is None:
        d_out = torch.zeros(36 * n, dtype=torch.float64, device="cuda")
    else:
        d_out = torch.from_numpy(np.ascontiguousarray(prev).reshape(-1).copy()).cuda()
    d_steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = _lib.lib().exg_pivot_inverse(device.handle, ctypes.c_void_p(d_in.data_ptr()), n, precision, form,
                                      int(prev is not None), ctypes.c_void_p(d_out.data_ptr()),
                                      ctypes.c_void_p(d_steps.data_ptr()))
    return rc, d_out.cpu().numpy().reshape(n, 6, 6), d_steps.cpu().numpy()


def residual(blocks, inv):
    eye = np.eye(6)
    return np.abs(np.einsum("bij,bjk->bik", blocks, inv) - eye).max(axis=(1, 2))


@pytest.mark.parametrize("n", [1, 37, 5000])
def test_thread_and_warp_forms_give_the_same_bits(device, n):
    blocks = pivot_like_blocks(n, seed=n)
    for precision in (PRECISION_F64, PRECISION_MIXED):
        rc0, x0, s0 = run(device, blocks, precision, 0)
        rc1, x1, s1 = run(device, blocks, precision, 1)
        _lib.check(rc0)
        _lib.check(rc1)
        assert np.array_equal(x0.view(np.uint64), x1.view(np.uint64)), precision
        assert np.array_equal(s0, s1)


def test_mixed_newton_schulz_error_and_steps(device):
    blocks = pivot_like_blocks(20000, seed=7)
    rc, x_ns, steps = run(device, blocks, PRECISION_MIXED, 0)
    _lib.check(rc)
    rc, x_gj, _ = run(device, blocks, PRECISION_F64, 0)
    _lib.check(rc)
    r_ns, r_gj = residual(blocks, x_ns), residual(blocks, x_gj)
    want = np.linalg.inv(blocks)
    rel_ns = np.abs(x_ns - want).max(axis=(1, 2)) / np.abs(want).max(axis=(1, 2))
    # every pivot-like block takes the Newton-Schulz path, in a handful of FP32 steps
    assert (steps >= 1).all() and steps.max() <= 16 and np.median(steps) <= 6, (steps.min(), steps.max())
    assert r_ns.max() <= 1e-11, r_ns.max()
    assert rel_ns.max() <= 1e-11, rel_ns.max()
    assert r_gj.max() <= 1e-12, r_gj.max()
    print(f"NS steps median {np.median(steps)}, max {steps.max()}; max|DX-I| NS {r_ns.max():.2e}, "
          f"GJ {r_gj.max():.2e}; rel err vs numpy NS {rel_ns.max():.2e}")


def test_ill_conditioned_block_falls_back_to_gauss_jordan(device):
    rng = np.random.default_rng(3)
    u, _ = np.linalg.qr(rng.normal(size=(6, 6)))
    v, _ = np.linalg.qr(rng.normal(size=(6, 6)))
    hard = u @ np.diag([1.0, 1.0, 1.0, 1e-3, 1e-6, 1e-9]) @ v.T  # condition 1e9: beyond FP32
    blocks = np.stack([pivot_like_blocks(1, seed=1)[0], hard])
    for form in (0, 1):
        rc, x, steps = run(device, blocks, PRECISION_MIXED, form)
        _lib.check(rc)
        assert steps[0] >= 1 and steps[1] == -1, steps
        want = np.linalg.inv(hard)
        assert np.abs(x[1] - want).max() <= 1e-5 * np.abs(want).max()


def test_singular_block_is_reported(device):
    blocks = pivot_like_blocks(3, seed=2)
    blocks[1] = 0.0
    for precision in (PRECISION_F64, PRECISION_MIXED):
        for form in (0, 1):
            rc, _, steps = run(device, blocks, precision, form)
            assert rc == -3, (precision, form, rc)  # EXG_ERR_FATAL
            if precision == PRECISION_MIXED:
                assert steps[1] == -1 and steps[0] >= 1


@pytest.mark.parametrize("change", [1e-9, 1e-5, 1e-2, 0.3])
def test_warm_start_from_the_previous_inverse(device, change):
    """The mixed path starts each solve after the first of a step from the node's previous
    inverse. A block that moved by `change` (relative, entrywise) from the one whose inverse is
    given: a tiny move takes the single FP64 correction (0 FP32 steps), a larger one FP32 steps
    seeded from the previous inverse, and a block that moved too far starts cold; every outcome
    is an accurate inverse, the same bits in both forms."""
    rng = np.random.default_rng(11)
    old = pivot_like_blocks(4000, seed=5)
    prev = np.linalg.inv(old)
    blocks = old * (1.0 + change * rng.uniform(-1.0, 1.0, size=old.shape))
    r0 = np.abs(np.eye(6) - np.einsum("bij,bjk->bik", blocks, prev)).max(axis=(1, 2))
    rc, x0, s0 = run(device, blocks, PRECISION_MIXED, 0, prev)
    _lib.check(rc)
    rc, x1, s1 = run(device, blocks, PRECISION_MIXED, 1, prev)
    _lib.check(rc)
    assert np.array_equal(x0.view(np.uint64), x1.view(np.uint64)) and np.array_equal(s0, s1)
    # the warm test is max|I - D X_prev| <= 1e-4 (margins keep the float boundary out of the check)
    assert (s0[r0 <= 0.9e-4] == 0).all()
    assert (s0[r0 > 1.1e-4] != 0).all()
    if change <= 1e-5:
        assert (s0 == 0).all()
    # a warm correction squares the previous residual (a 6x6 product: within 6 r0^2); the FP32 path
    # ends at its floor, squared
    res = residual(blocks, x0)
    warm = s0 == 0
    assert (res[warm] <= 6.0 * r0[warm] ** 2 + 1e-13).all(), (res[warm] / r0[warm] ** 2).max()
    assert res[~warm].max(initial=0.0) <= (1e-9 if change <= 1e-2 else 1e-6), res[~warm].max(initial=0.0)


@pytest.mark.parametrize("schedule", ["island", "wave"])
def test_ns_pivots_step_a_tree_like_gauss_jordan_and_the_oracle(device, oracle, schedule):
    """A mixed-precision random tree stepped with Newton-Schulz pivot inverses ends where the same
    tree with Gauss-Jordan pivots does and where the f64 oracle does (both solves converge the same
    Newton iteration to the same tolerance)."""
    from exgame_b200 import scenarios
    from exgame_b200.abi import NEWTON, step_params
    from test_gpu_parity import state_error
    bodies, joints = scenarios.tree_world(600, seed=73)
    out = {}
    for ns in (False, True):
        params = step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10, exact_jacobian=True,
                             ns_pivot=ns)
        w = _lib.DeviceWorld(device, bodies, joints, params)
        w.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 1 << 20 if schedule == "island" else 1)
        w.step(40)
        out[ns] = w.bodies()
        assert w.stats()["fatal"] == 0
        w.close()
    q = step_params(integrator=NEWTON, precision=0, dt=1e-2, tol=1e-10, exact_jacobian=True)
    ow = oracle.OracleWorld(bodies, joints, q)
    ow.step(40)
    pe, me = state_error(out[False], out[True])
    assert pe < 1e-11 and me < 1e-9, (pe, me)
    pe, me = state_error(ow.bodies(), out[True])
    assert pe < 1e-9 and me < 1e-7, (pe, me)


def test_ns_pivots_on_a_curtain_match_the_oracle(device, oracle):
    """An island with dynamic cycles (the block-LU solve) with Newton-Schulz pivot inverses."""
    from exgame_b200 import scenarios
    from test_gpu_parity import state_error
    bodies, joints, params = scenarios.cloth_world(6, 8, tol=1e-10, precision=PRECISION_MIXED)
    params["newton_flags"] |= 2  # EXG_NEWTON_NS_PIVOT
    w = _lib.DeviceWorld(device, bodies, joints, params)
    w.step(30)
    got = w.bodies()
    w.close()
    q = params.copy()
    q["precision"] = 0
    q["newton_flags"] = 0
    ow = oracle.OracleWorld(bodies, joints, q)
    ow.step(30)
    pe, me = state_error(ow.bodies(), got)
    assert pe < 1e-8 and me < 1e-6, (pe, me)


def test_worlds_with_and_without_ns_pivots_in_one_batch_step_as_alone(device):
    """One world asking for Newton-Schulz pivots makes the batch launch the kernels that carry them;
    the other worlds still take Gauss-Jordan inside them. Every world of such a batch (both
    schedules) ends bit for bit as it does alone."""
    from exgame_b200 import scenarios
    from exgame_b200.abi import NEWTON, step_params
    worlds = []
    for k, (n, ns) in enumerate([(60, True), (60, False), (900, True), (900, False), (12, False)]):
        b, j = scenarios.tree_world(n, seed=500 + k)
        worlds.append((b, j, step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10,
                                         exact_jacobian=True, ns_pivot=ns)))
    batch = _lib.DeviceBatch(device, worlds)
    batch.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 32)
    batch.step(4)
    for k, (b, j, p) in enumerate(worlds):
        alone = _lib.DeviceWorld(device, b, j, p)
        alone.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 32)
        alone.step(4)
        got, want = batch.world_bodies(k), alone.bodies()
        assert np.array_equal(got["pose"], want["pose"]) and np.array_equal(got["momentum"], want["momentum"]), k
        alone.close()
    batch.close()
