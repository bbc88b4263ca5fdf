"""Autotuner of the device's launch shapes.

Each tuned quantity changes how work is spread over the SMs, never the arithmetic: the gravity
items and their j-ranges depend on a world's size alone, the wave schedule's per-item work and
reduction orders are fixed, and the island kernel and the wave give identical results. So the
tuner may pick whatever runs fastest on this GPU, and results stay bit-identical to untuned runs
(tested). It times each candidate on small synthetic workloads through the public API (device
time from the library's own event profiler), keeps the fastest, and leaves it set on the device:

  gravity CTAs per SM   persistent one-warp CTAs of the mixed gravity kernel
  wave blocks per SM    grid cap of the wave schedule's data kernels
  wave threshold        dynamic bodies from which an island takes the wave schedule
  narrow level          elimination levels up to this many nodes (over all wave islands) take one
                        warp per node, wider ones one thread per node; tuned on a batch of trees
                        large enough to have levels of both kinds
"""
import numpy as np

from . import _lib, scenarios
from .abi import GRAVITY_PLUMMER, JOINT_DTYPE, LIE_EULER, NEWTON, PRECISION_MIXED, step_params

GRAVITY_CTAS = (8, 12, 16, 21, 32)
WAVE_BLOCKS = (4, 8, 16)
WAVE_THRESHOLDS = (8, 16, 32, 256)
NARROW_LEVELS = (8192, 32768, 1 << 30)


def _time(dev, kinds, world, steps):
    world.step(1)  # structure synced, graphs captured
    dev.profile(True)
    world.step(steps)
    ms = sum(dev.profile_read(k)[0] for k in kinds)
    dev.profile(False)
    return ms / steps


def _best(d):
    return min(d, key=d.get)


def _tune_on(dev, world, out, steps):
    """Every knob timed on the caller's own handle, one after another, each left at its best."""
    D = _lib.Device
    kinds = (D.PROF_NEWTON, D.PROF_NEWTON_WAVE)
    for c in GRAVITY_CTAS:
        dev.set_tuning(D.TUNE_GRAVITY_CTAS_PER_SM, c)
        out["gravity_ctas_per_sm"][c] = _time(dev, (D.PROF_GRAVITY,), world, steps)
    dev.set_tuning(D.TUNE_GRAVITY_CTAS_PER_SM, _best(out["gravity_ctas_per_sm"]))
    for b in WAVE_BLOCKS:
        dev.set_tuning(D.TUNE_WAVE_BLOCKS_PER_SM, b)
        out["wave_blocks_per_sm"][b] = _time(dev, kinds, world, steps)
    dev.set_tuning(D.TUNE_WAVE_BLOCKS_PER_SM, _best(out["wave_blocks_per_sm"]))
    for t in WAVE_THRESHOLDS:
        world.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, t)
        out["wave_min_bodies"][t] = _time(dev, kinds, world, steps)
    best_t = _best(out["wave_min_bodies"])
    world.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, best_t)
    dev.set_tuning(D.TUNE_WAVE_MIN_BODIES, best_t)
    for nl in NARROW_LEVELS:
        dev.set_tuning(D.TUNE_WAVE_NARROW_LEVEL, nl)
        out["wave_narrow_level"][nl] = _time(dev, kinds, world, steps)
    dev.set_tuning(D.TUNE_WAVE_NARROW_LEVEL, _best(out["wave_narrow_level"]))


def autotune(dev, gravity_bodies=32768, trees=24, tree_bodies=1500, steps=3, seed=11, workload=None):
    """Measure the candidates on `dev`, set the fastest, return the choices and their timings.

    With `workload` (an open DeviceWorld or DeviceBatch) every candidate is timed on that handle's
    own steps, which advance its state, and its wave threshold is left at the best candidate;
    otherwise on the synthetic worlds above."""
    D = _lib.Device
    out = {"gravity_ctas_per_sm": {}, "wave_blocks_per_sm": {}, "wave_min_bodies": {}, "wave_narrow_level": {}}
    if workload is not None:
        _tune_on(dev, workload, out, steps)
        return {"gravity_ctas_per_sm": _best(out["gravity_ctas_per_sm"]),
                "wave_blocks_per_sm": _best(out["wave_blocks_per_sm"]),
                "wave_min_bodies": _best(out["wave_min_bodies"]),
                "wave_narrow_level": _best(out["wave_narrow_level"]), "timed_on": "workload",
                "ms": {k: {str(c): round(v, 4) for c, v in d.items()} for k, d in out.items()}}
    g = scenarios.gravity_world(gravity_bodies, 1000.0, seed=seed)
    gw = _lib.DeviceWorld(dev, g, np.zeros(0, dtype=JOINT_DTYPE),
                          step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, precision=PRECISION_MIXED,
                                      softening=0.05, dt=1e-3))
    for c in GRAVITY_CTAS:
        dev.set_tuning(D.TUNE_GRAVITY_CTAS_PER_SM, c)
        out["gravity_ctas_per_sm"][c] = _time(dev, (D.PROF_GRAVITY,), gw, steps)
    gw.close()
    best_g = min(out["gravity_ctas_per_sm"], key=out["gravity_ctas_per_sm"].get)
    dev.set_tuning(D.TUNE_GRAVITY_CTAS_PER_SM, best_g)

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(16), np.log(tree_bodies), size=trees)).astype(int)
    p = step_params(integrator=NEWTON, precision=PRECISION_MIXED, dt=1e-2, tol=1e-10, exact_jacobian=True)
    worlds = [(*scenarios.tree_world(int(n), seed=seed + k), p) for k, n in enumerate(sizes)]
    batch = _lib.DeviceBatch(dev, worlds)
    kinds = (D.PROF_NEWTON, D.PROF_NEWTON_WAVE)
    batch.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 1)
    for b in WAVE_BLOCKS:
        dev.set_tuning(D.TUNE_WAVE_BLOCKS_PER_SM, b)
        out["wave_blocks_per_sm"][b] = _time(dev, kinds, batch, steps)
    best_b = min(out["wave_blocks_per_sm"], key=out["wave_blocks_per_sm"].get)
    dev.set_tuning(D.TUNE_WAVE_BLOCKS_PER_SM, best_b)
    for t in WAVE_THRESHOLDS:
        batch.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, t)
        out["wave_min_bodies"][t] = _time(dev, kinds, batch, steps)
    batch.close()
    best_t = min(out["wave_min_bodies"], key=out["wave_min_bodies"].get)
    dev.set_tuning(D.TUNE_WAVE_MIN_BODIES, best_t)
    # wide levels need many large trees at once: 48 trees of 2048 bodies
    wide = [(*scenarios.tree_world(2048, seed=seed + 100 + k), p) for k in range(48)]
    wb = _lib.DeviceBatch(dev, wide)
    wb.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, best_t)
    for nl in NARROW_LEVELS:
        dev.set_tuning(D.TUNE_WAVE_NARROW_LEVEL, nl)
        out["wave_narrow_level"][nl] = _time(dev, kinds, wb, steps)
    wb.close()
    best_n = min(out["wave_narrow_level"], key=out["wave_narrow_level"].get)
    dev.set_tuning(D.TUNE_WAVE_NARROW_LEVEL, best_n)
    return {"gravity_ctas_per_sm": best_g, "wave_blocks_per_sm": best_b, "wave_min_bodies": best_t,
            "wave_narrow_level": best_n,
            "ms": {k: {str(c): round(v, 4) for c, v in d.items()} for k, d in out.items()}}
