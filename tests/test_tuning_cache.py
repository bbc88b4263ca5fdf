"""The autotuner's per-GPU, per-shape cache (host logic, no GPU): a miss times the candidates and
stores the choices, a hit sets them without timing, the bucket separates workload shapes, and a
corrupt, other-version or out-of-candidate file is never trusted."""
import json

import numpy as np
import pytest

from exgame_b200 import _lib, autotune
from exgame_b200.abi import LIE_EULER, NEWTON, NEWTON_NS_PIVOT, PRECISION_F64, PRECISION_MIXED, STEP_PARAMS_DTYPE


class FakeDevice:
    ordinal = 0

    def __init__(self):
        self.tuning = {}

    def set_tuning(self, key, value):
        self.tuning[key] = value

    def get_tuning(self, key):
        return self.tuning[key]


class FakeBatch:
    def __init__(self, counts, integrators, precision=PRECISION_MIXED, flags=0):
        self.counts = np.asarray(counts, dtype=np.int32)
        self.n = int(self.counts.sum())
        self.params = np.zeros(len(counts), dtype=STEP_PARAMS_DTYPE)
        self.params["integrator"] = integrators
        self.params["precision"] = precision
        self.params["newton_flags"] = flags
        self.options = {}

    def set_option(self, key, value):
        self.options[key] = value


# timings the fake measurement reports: the best of each knob is a fixed, non-default candidate
FAKE_MS = {"gravity_ctas_per_sm": {8: 3.0, 12: 2.0, 16: 2.5, 21: 4.0, 32: 5.0},
           "wave_blocks_per_sm": {4: 1.0, 8: 2.0, 16: 3.0},
           "wave_min_bodies": {8: 4.0, 16: 3.0, 32: 3.5, 256: 9.0},
           "wave_narrow_level": {8192: 2.0, 32768: 1.5, 1 << 30: 3.0}}


@pytest.fixture
def timed(monkeypatch):
    calls = []

    def fake_tune_on(dev, world, out, steps):
        calls.append(world)
        for k, d in FAKE_MS.items():
            out[k].update(d)
        for name, key, _ in autotune.KNOBS:
            dev.set_tuning(key, min(FAKE_MS[name], key=FAKE_MS[name].get))
        world.set_option(_lib.DeviceWorld.OPT_WAVE_MIN_BODIES, 16)

    monkeypatch.setattr(autotune, "_tune_on", fake_tune_on)
    return calls


BEST = {"gravity_ctas_per_sm": 12, "wave_blocks_per_sm": 4, "wave_min_bodies": 16, "wave_narrow_level": 32768}


def batch():
    return FakeBatch([8, 300, 2000, 8192], [LIE_EULER, NEWTON, NEWTON, LIE_EULER])


def test_miss_times_and_stores_then_hit_sets_without_timing(tmp_path, timed):
    path = tmp_path / "tuning.json"
    dev = FakeDevice()
    r1 = autotune.autotune(dev, workload=batch(), cache=str(path), device_key="gpuA")
    assert len(timed) == 1 and r1["timed_on"] == "workload"
    assert {k: r1[k] for k in BEST} == BEST
    doc = json.loads(path.read_text())
    assert doc["version"] == autotune.CACHE_VERSION
    (entry_key, entry), = doc["entries"].items()
    assert entry_key == "gpuA|" + autotune.workload_bucket(batch())
    assert {k: entry[k] for k in BEST} == BEST and "ms" in entry

    dev2, w2 = FakeDevice(), batch()
    r2 = autotune.autotune(dev2, workload=w2, cache=autotune.TuningCache(path), device_key="gpuA")
    assert len(timed) == 1, "a hit must not time anything"
    assert r2["timed_on"] == "cache" and {k: r2[k] for k in BEST} == BEST
    assert dev2.tuning == {key: BEST[name] for name, key, _ in autotune.KNOBS}
    assert w2.options == {_lib.DeviceWorld.OPT_WAVE_MIN_BODIES: 16}


def test_other_gpu_or_shape_misses(tmp_path, timed):
    path = str(tmp_path / "tuning.json")
    autotune.autotune(FakeDevice(), workload=batch(), cache=path, device_key="gpuA")
    autotune.autotune(FakeDevice(), workload=batch(), cache=path, device_key="gpuB")
    assert len(timed) == 2
    other = FakeBatch([8, 300, 2000, 8192] * 4, [LIE_EULER, NEWTON, NEWTON, LIE_EULER] * 4)
    autotune.autotune(FakeDevice(), workload=other, cache=path, device_key="gpuA")
    assert len(timed) == 3
    assert len(autotune.TuningCache(path).entries()) == 3


def test_no_cache_always_times(timed):
    autotune.autotune(FakeDevice(), workload=batch())
    autotune.autotune(FakeDevice(), workload=batch())
    assert len(timed) == 2


@pytest.mark.parametrize("content", ["{not json", json.dumps([1, 2]), json.dumps({"version": 999, "entries": {}}),
                                     json.dumps({"version": 1, "entries": "x"})])
def test_unreadable_or_other_version_file_is_ignored_and_replaced(tmp_path, timed, content):
    path = tmp_path / "tuning.json"
    path.write_text(content)
    r = autotune.autotune(FakeDevice(), workload=batch(), cache=str(path), device_key="gpuA")
    assert len(timed) == 1 and r["timed_on"] == "workload"
    assert json.loads(path.read_text())["version"] == autotune.CACHE_VERSION


@pytest.mark.parametrize("bad", [{"gravity_ctas_per_sm": 7}, {"wave_blocks_per_sm": "8"},
                                 {"wave_min_bodies": True}, {"wave_narrow_level": None}])
def test_entry_with_a_non_candidate_value_is_not_trusted(tmp_path, timed, bad):
    path = tmp_path / "tuning.json"
    entry = dict(BEST, **bad)
    key = "gpuA|" + autotune.workload_bucket(batch())
    path.write_text(json.dumps({"version": autotune.CACHE_VERSION, "entries": {key: entry}}))
    dev = FakeDevice()
    r = autotune.autotune(dev, workload=batch(), cache=str(path), device_key="gpuA")
    assert len(timed) == 1 and r["timed_on"] == "workload"
    assert autotune.TuningCache(path).get("gpuA", autotune.workload_bucket(batch())) == BEST


def test_missing_folder_is_created_and_no_temporary_left(tmp_path, timed):
    path = tmp_path / "a" / "b" / "tuning.json"
    autotune.autotune(FakeDevice(), workload=batch(), cache=str(path), device_key="gpuA")
    assert path.exists()
    assert sorted(p.name for p in path.parent.iterdir()) == ["tuning.json", "tuning.json.lock"]


def test_bucket_edges():
    b = autotune.shape_bucket
    base = b([100, 200, 300], [NEWTON, NEWTON, LIE_EULER], [1, 1, 1])
    # same powers of two in world count, total and largest: same bucket
    assert b([110, 210, 310], [NEWTON, NEWTON, LIE_EULER], [1, 1, 1]) == base
    # the largest world crosses 512
    assert b([100, 200, 600], [NEWTON, NEWTON, LIE_EULER], [1, 1, 1]) != base
    # twice the worlds
    assert b([100, 200, 300] * 2, [NEWTON, NEWTON, LIE_EULER] * 2, [1] * 6) != base
    # implicit share 2/3 -> 1/3
    assert b([100, 200, 300], [NEWTON, LIE_EULER, LIE_EULER], [1, 1, 1]) != base
    # precision and pivot form are exact parts of the key
    assert b([100, 200, 300], [NEWTON, NEWTON, LIE_EULER], [PRECISION_F64] * 3) != base
    assert b([100, 200, 300], [NEWTON, NEWTON, LIE_EULER], [1, 1, 1], [NEWTON_NS_PIVOT] * 3) != base
    # order of worlds does not matter
    assert b([300, 100, 200], [LIE_EULER, NEWTON, NEWTON], [1, 1, 1]) == base
    with pytest.raises(ValueError):
        b([1, 2], [NEWTON], [1, 1])


def test_single_world_bucket():
    w = FakeBatch([5000], [NEWTON])
    del w.counts
    w.params = w.params[0]
    assert autotune.workload_bucket(w) == autotune.shape_bucket([5000], [NEWTON], [PRECISION_MIXED])


def test_library_build_id_tracks_file_content(tmp_path):
    p = tmp_path / "lib.so"
    p.write_bytes(b"a" * 100)
    a = autotune.library_build_id(str(p))
    assert a == autotune.library_build_id(str(p)) and len(a) == 12
    p.write_bytes(b"b" * 101)
    assert autotune.library_build_id(str(p)) != a


def _put_many(path, worker, n):
    cache = autotune.TuningCache(path)
    for k in range(n):
        cache.put(f"gpu{worker}", f"bucket{k}", BEST)


def test_concurrent_writers_keep_every_entry(tmp_path):
    """Processes writing different buckets at once (ranks sharing one file) lose none of them."""
    import multiprocessing as mp
    path = str(tmp_path / "tuning.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_put_many, args=(path, w, 15)) for w in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    entries = autotune.TuningCache(path).entries()
    assert len(entries) == 60
    assert all(autotune.TuningCache(path).get(f"gpu{w}", f"bucket{k}") == BEST for w in range(4) for k in range(15))


def test_unwritable_cache_keeps_the_measured_choices(tmp_path, timed):
    """A cache path that cannot be written (its folder is a file) does not undo the tuning."""
    blocker = tmp_path / "not_a_folder"
    blocker.write_text("x")
    dev = FakeDevice()
    r = autotune.autotune(dev, workload=batch(), cache=str(blocker / "tuning.json"), device_key="gpuA")
    assert r["timed_on"] == "workload" and "cache_error" in r
    assert {k: r[k] for k in BEST} == BEST
    assert dev.tuning == {key: BEST[name] for name, key, _ in autotune.KNOBS}
