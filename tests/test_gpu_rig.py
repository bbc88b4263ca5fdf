"""The hitchcock camera rig on the device against the oracle: the host moves every rig's kinematic
tracker before each step through the C ABI (exg_world_get_state / exg_world_set_state), as the
reference's TargetTracker::pre_step does (crates/hitchcock/src/camera.rs:55-76), including a
retarget that teleports the tracker; the device state matches the f64 oracle's after every
segment, on both Newton schedules, in FP64 and in mixed precision."""
import numpy as np
import pytest

from exgame_b200 import _lib, scenarios
from exgame_b200.abi import PRECISION_MIXED
from test_gpu_parity import state_error
from test_rig import rig_target, state_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,schedule", [(0, "island"), (0, "wave"), (PRECISION_MIXED, "wave")])
def test_rig_tracks_like_the_oracle(device, oracle, precision, schedule):
    n = 8
    b, j, p = scenarios.camera_rig_world(n, r_object=2.0, linear=1.0, precision=precision)
    q = p.copy()
    q["precision"] = 0
    ow = oracle.OracleWorld(b, j, q)
    dw = _lib.DeviceWorld(device, b, j, p)
    dw.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 1 if schedule == "wave" else 1 << 20)
    dt = float(p["dt"])
    worst = 0.0
    for s in range(300):
        centres, vel = rig_target(s * dt, n)
        dw.set_state(scenarios.track_targets(dw.state(), n, centres, vel))
        cur = ow.bodies()
        st = scenarios.track_targets(state_of(cur), n, centres, vel)
        cur["pose"], cur["momentum"] = st[:, :8], st[:, 8:]
        ow.set_state(cur)
        dw.step(1)
        ow.step(1)
        if s % 50 == 49:
            pe, me = state_error(ow.bodies(), dw.bodies())
            worst = max(worst, pe)
            assert pe < (1e-9 if precision == 0 else 1e-7) and me < (1e-7 if precision == 0 else 1e-5), (s, pe, me)
    assert dw.stats()["fatal"] == 0
    dw.close()
