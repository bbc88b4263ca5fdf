"""The oracle at large world offsets (the property of crates/newton/tests/precision_seam.rs): the
reference's five-body spring chain translated by 2^10, 2^20 and 2^30 on every axis keeps its shape
after 20 implicit steps to within 64 FP64 spacings at the offset, in the same spans and Newton
iterations as at the origin, because each island steps in a frame anchored near its centre of
mass on a 1024 grid (the offsets are on the grid, so the chain sits in its frame as at the
origin)."""
import numpy as np
import pytest

from exgame_b200 import motors_np
from exgame_b200.abi import GRAVITY_OFF, NEWTON, step_params
from test_gpu_seam import DT, N, STEPS, grid_chain


def oracle_run(oracle, offset):
    b, j = grid_chain(offset)
    p = step_params(integrator=NEWTON, gravity_law=GRAVITY_OFF, dt=DT, tol=1e-10, field=(0.0, 0.0, -9.81))
    ow = oracle.OracleWorld(b, j, p)
    ow.step(STEPS)
    out = ow.bodies()
    pos = motors_np.apply_point_n(out["pose"], np.zeros((N, 3)))
    return pos - pos[0], ow.island_stats()


@pytest.mark.parametrize("offset", [2.0 ** 10, 2.0 ** 20, 2.0 ** 30])
def test_oracle_keeps_the_shape_far_from_the_origin(oracle, offset):
    ref, ref_stats = oracle_run(oracle, 0.0)
    far, far_stats = oracle_run(oracle, offset)
    assert np.abs(far - ref).max() <= 64.0 * np.spacing(offset)
    assert far_stats == ref_stats  # no extra sub-division or Newton iterations far away
