"""Typed slot storage on the device (exg_storage_* / exg_slot_*), restating the reference's own
storage tests (crates/aristotle/src/world.rs:656-900): insert and read back, write through a key,
stale keys after free, the lowest free slot reused first, the high-water mark, growth that keeps
every index and moves the generation once per reallocation, reuse that does not grow; plus the
batched forms and the one-writer refusal of a batch that names one slot twice."""
import numpy as np
import pytest

from exgame_b200 import _lib

pytestmark = pytest.mark.gpu

VEC3 = np.dtype([("x", np.float32), ("y", np.float32), ("z", np.float32)])


def test_insert_read_write(device):
    st = _lib.SlotStorage(device, np.uint32, 100)
    k, k2 = st.alloc(42), st.alloc(27)
    assert st.read(k) == 42 and st.read(k2) == 27
    st.write(k, 117)
    assert st.read(k) == 117 and st.read(k2) == 27
    st.free(k)
    assert st.read(k2) == 27
    st.close()


def test_types_do_not_collide(device):
    ints, vecs = _lib.SlotStorage(device, np.uint32, 8), _lib.SlotStorage(device, VEC3, 8)
    a, b = ints.alloc(7), ints.alloc(8)
    v = vecs.alloc(np.array((1.0, 2.0, 3.0), dtype=VEC3))
    assert ints.read(a) == 7 and ints.read(b) == 8
    assert tuple(vecs.read(v).tolist()) == (1.0, 2.0, 3.0)
    ints.close()
    vecs.close()


def test_stale_key_is_refused_and_slot_reused_with_new_generation(device):
    st = _lib.SlotStorage(device, np.uint32, 100)
    key = st.alloc(100)
    st.free(key)
    with pytest.raises(_lib.ExgError) as e:
        st.read(key)
    assert e.value.status == -20
    key2 = st.alloc(200)
    assert key2["index"] == key["index"] and key2["generation"] != key["generation"]
    with pytest.raises(_lib.ExgError):
        st.read(key)
    with pytest.raises(_lib.ExgError):
        st.write(key, 1)
    with pytest.raises(_lib.ExgError):  # freeing twice is refused
        st.free(key)
    assert st.read(key2) == 200
    st.close()


def test_lowest_free_slot_first_and_high_water_mark(device):
    st = _lib.SlotStorage(device, np.uint32, 100)
    k = [st.alloc(i) for i in range(4)]
    for i in (1, 3, 0):  # out of order
        st.free(k[i])
    assert st.alloc(10)["index"] == k[0]["index"]
    assert st.alloc(11)["index"] == k[1]["index"]
    assert st.alloc(13)["index"] == k[3]["index"]
    assert st.read(k[2]) == 2
    assert st.alloc(14)["index"] == 4
    info = st.info()
    assert info["len"] == 5 and info["live"] == 5
    st.close()


def test_growth_keeps_indices_and_bumps_generation_per_reallocation(device):
    st = _lib.SlotStorage(device, np.uint32, 2)
    buf0 = int(st.info()["buffer"])
    keys = [st.alloc(i * 10) for i in range(9)]
    info = st.info()
    assert info["capacity"] >= 9 and info["generation"] == 3  # 2 -> 4 -> 8 -> 16
    assert int(info["buffer"]) != buf0
    for i, k in enumerate(keys):
        assert k["index"] == i and st.read(k) == i * 10
    st.write(keys[8], 7)
    assert st.read(keys[8]) == 7
    st.close()


def test_reuse_does_not_grow(device):
    st = _lib.SlotStorage(device, np.uint32, 2)
    k0 = st.alloc(1)
    st.alloc(2)
    st.free(k0)
    st.alloc(3)
    info = st.info()
    assert info["capacity"] == 2 and info["generation"] == 0
    st.close()


def test_batched_read_write_and_one_writer_refusal(device):
    st = _lib.SlotStorage(device, VEC3, 16)
    vals = np.zeros(40, dtype=VEC3)
    vals["x"] = np.arange(40)
    keys = np.array([st.alloc(v) for v in vals], dtype=_lib.SLOT_KEY_DTYPE)
    assert np.array_equal(st.read_n(keys)["x"], vals["x"])
    pick = keys[[3, 17, 0, 39]]
    new = np.zeros(4, dtype=VEC3)
    new["y"] = [1, 2, 3, 4]
    st.write_n(pick, new)
    assert np.array_equal(st.read_n(pick)["y"], new["y"])
    twice = keys[[5, 6, 5]]
    before = st.read_n(keys)
    with pytest.raises(_lib.ExgError) as e:
        st.write_n(twice, np.ones(3, dtype=VEC3))
    assert e.value.status == -5 and "second writer" in str(e.value)
    assert np.array_equal(st.read_n(keys), before)  # nothing written
    st.free(keys[9])
    with pytest.raises(_lib.ExgError):  # a stale key refuses the whole batch
        st.write_n(keys[[8, 9]], np.ones(2, dtype=VEC3))
    assert np.array_equal(st.read_n(keys[[8]]), before[[8]])
    st.close()
