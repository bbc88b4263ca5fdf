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

The choices can be kept in a TuningCache file per GPU and workload shape bucket (the end of this
module), so that a process whose batch falls in a bucket already tuned on this GPU sets them
without timing.
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


def autotune(dev, gravity_bodies=32768, trees=24, tree_bodies=1500, steps=3, seed=11, workload=None, cache=None,
             device_key=None):
    """Measure the candidates on `dev`, set the fastest, return the choices and their timings.

    With `workload` (an open DeviceWorld or DeviceBatch) every candidate is timed on that handle's
    own steps, which advance its state, and its wave threshold is left at the best candidate;
    otherwise on the synthetic worlds above.

    With `cache` (a TuningCache or a file path) the choices are looked up first under this GPU's
    key and the workload's shape bucket: a hit sets them without timing anything (the workload's
    state is left alone) and returns them with `timed_on` "cache"; a miss measures as above and
    stores the result (a file that cannot be written leaves the measured choices set and is
    reported under `cache_error`). `device_key` overrides the GPU's key (its name, SM count and the
    library build)."""
    if cache is None:
        return _measure(dev, gravity_bodies, trees, tree_bodies, steps, seed, workload)
    if not isinstance(cache, TuningCache):
        cache = TuningCache(cache)
    key = device_key if device_key is not None else gpu_key(dev)
    if workload is not None:
        bucket = workload_bucket(workload)
    else:
        bucket = f"synthetic.g{gravity_bodies}.t{trees}x{tree_bodies}.s{seed}"
    hit = cache.get(key, bucket)
    if hit is not None:
        apply(dev, hit, workload)
        return dict(hit, timed_on="cache", bucket=bucket)
    res = _measure(dev, gravity_bodies, trees, tree_bodies, steps, seed, workload)
    try:
        cache.put(key, bucket, res)
    except OSError as e:  # the choices are measured and set; only keeping them failed
        return dict(res, bucket=bucket, cache_error=f"{type(e).__name__}: {e}")
    return dict(res, bucket=bucket)


def _measure(dev, gravity_bodies, trees, tree_bodies, steps, seed, workload):
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


# ── tuning cache per GPU and workload shape ──
#
# A serving host sees the same few batch shapes again and again; timing the candidates costs a
# few seconds of steps each time. The cache keeps the chosen values per (GPU, shape bucket) in a
# JSON file, so a later process with a batch in the same bucket sets them without timing. Bucket
# edges are powers of two in world count, total bodies and largest world, eighths of the implicit
# share of worlds, and the exact set of precisions and pivot forms: the quantities the knobs'
# best values depend on (the gravity grid on the tile count, the wave knobs on the implicit
# islands' sizes). A stale or unreadable file is ignored, never trusted.

CACHE_VERSION = 1
KNOBS = (("gravity_ctas_per_sm", 1, GRAVITY_CTAS), ("wave_blocks_per_sm", 2, WAVE_BLOCKS),
         ("wave_min_bodies", 3, WAVE_THRESHOLDS), ("wave_narrow_level", 4, NARROW_LEVELS))
_build_ids = {}


def _log2_bucket(n):
    return int(n).bit_length() - 1 if n > 0 else -1


def shape_bucket(body_counts, integrators, precisions, flags=None):
    """The cache key of a batch: log2 buckets of its world count, total and largest body count,
    the implicit worlds' share in eighths, and the precisions and Newton flags in use."""
    counts = np.asarray(body_counts, dtype=np.int64).ravel()
    integ = np.asarray(integrators).ravel()
    prec = sorted({int(p) for p in np.asarray(precisions).ravel()})
    fl = sorted({int(f) for f in np.asarray(flags if flags is not None else [0] * len(counts)).ravel()})
    if len(counts) != len(integ) or len(counts) != len(np.asarray(precisions).ravel()):
        raise ValueError("body_counts, integrators and precisions need one entry per world")
    n = len(counts)
    eighths = int(round(8.0 * float((integ == NEWTON).sum()) / n)) if n else 0
    return (f"w{_log2_bucket(n)}.b{_log2_bucket(int(counts.sum()))}.m{_log2_bucket(int(counts.max()) if n else 0)}"
            f".i{eighths}.p{'-'.join(map(str, prec))}.f{'-'.join(map(str, fl))}")


def workload_bucket(world):
    """shape_bucket of an open DeviceWorld (one world) or DeviceBatch."""
    params = np.atleast_1d(world.params)
    counts = getattr(world, "counts", None)
    if counts is None:
        counts = [world.n]
    return shape_bucket(counts, params["integrator"], params["precision"], params["newton_flags"])


def library_build_id(path=None):
    """A short hash of the loaded library file: tuned values belong to the kernels they were timed on."""
    import hashlib
    import os
    path = path or _lib.LIB_PATH
    st = os.stat(path)
    key = (path, st.st_size, st.st_mtime_ns)
    if key not in _build_ids:
        h = hashlib.sha1()
        with open(path, "rb") as f:
            for chunk in iter(lambda: f.read(1 << 20), b""):
                h.update(chunk)
        _build_ids[key] = h.hexdigest()[:12]
    return _build_ids[key]


def gpu_key(dev):
    """This GPU's cache key: its name and SM count (from the CUDA runtime, through torch) and the
    library build."""
    import torch
    p = torch.cuda.get_device_properties(dev.ordinal)
    return f"{p.name}/{p.multi_processor_count}sm/{library_build_id()}"


def apply(dev, choice, workload=None):
    """Set a cached choice on the device (and the workload's wave threshold, as tuning does)."""
    for name, key, _ in KNOBS:
        dev.set_tuning(key, int(choice[name]))
    if workload is not None:
        workload.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, int(choice["wave_min_bodies"]))


class TuningCache:
    """The JSON file of tuned choices: {"version": 1, "entries": {"<gpu>|<bucket>": {knob: value, ...}}}.

    Reads tolerate a missing, unreadable or other-version file (empty cache) and drop entries whose
    values are not candidates of this tuner. A write holds an exclusive lock on a sidecar file
    (`<path>.lock`, flock) across its read, merge and write, and replaces the file through a
    temporary file and an atomic rename: concurrent processes (one per rank) keep each other's
    entries, and a reader never sees half a file."""

    def __init__(self, path):
        self.path = str(path)

    def _load(self):
        import json
        try:
            with open(self.path) as f:
                doc = json.load(f)
        except (OSError, ValueError):
            return {}
        if not isinstance(doc, dict) or doc.get("version") != CACHE_VERSION or not isinstance(doc.get("entries"), dict):
            return {}
        return doc["entries"]

    @staticmethod
    def _valid(entry):
        if not isinstance(entry, dict):
            return False
        for name, _, candidates in KNOBS:
            v = entry.get(name)
            if isinstance(v, bool) or not isinstance(v, int) or v not in candidates:
                return False
        return True

    def get(self, gpu, bucket):
        entry = self._load().get(f"{gpu}|{bucket}")
        if not self._valid(entry):
            return None
        return {name: entry[name] for name, _, _ in KNOBS}

    def put(self, gpu, bucket, result):
        import json
        import os
        import tempfile
        import fcntl
        entry = {name: int(result[name]) for name, _, _ in KNOBS}
        if "ms" in result:
            entry["ms"] = result["ms"]
        folder = os.path.dirname(os.path.abspath(self.path))
        os.makedirs(folder, exist_ok=True)
        with open(self.path + ".lock", "a") as lock:
            fcntl.flock(lock, fcntl.LOCK_EX)
            try:
                entries = self._load()
                entries[f"{gpu}|{bucket}"] = entry
                fd, tmp = tempfile.mkstemp(prefix=".tuning.", dir=folder)
                try:
                    with os.fdopen(fd, "w") as f:
                        json.dump({"version": CACHE_VERSION, "entries": entries}, f, indent=1, sort_keys=True)
                    os.replace(tmp, self.path)
                except BaseException:
                    if os.path.exists(tmp):
                        os.unlink(tmp)
                    raise
            finally:
                fcntl.flock(lock, fcntl.LOCK_UN)

    def entries(self):
        return dict(self._load())
