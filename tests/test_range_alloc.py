"""The pools' range allocator (exgame_b200/csrc/range_alloc.hpp) compiled for the host and checked
against a model occupancy map under random admissions and releases: ranges never overlap, stay
inside the capacity, first fit takes the lowest free offset, freed ranges coalesce, growth appends
free space, and the launch extent (one past the highest used element) is exact."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "range_alloc_host.cpp")
OUT = os.path.join(HERE, "native", "_build", "librange_alloc_host.so")


@pytest.fixture(scope="module")
def ra():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", OUT, SRC], check=True)
    L = ctypes.CDLL(OUT)
    L.ra_new.restype = ctypes.c_void_p
    L.ra_new.argtypes = [ctypes.c_longlong]
    for fn in ("ra_alloc",):
        getattr(L, fn).restype = ctypes.c_longlong
        getattr(L, fn).argtypes = [ctypes.c_void_p, ctypes.c_longlong]
    L.ra_release.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong]
    L.ra_alloc_at.restype = ctypes.c_int
    L.ra_alloc_at.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong]
    L.ra_grow.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
    for fn in ("ra_capacity", "ra_largest_free", "ra_used_end"):
        getattr(L, fn).restype = ctypes.c_longlong
        getattr(L, fn).argtypes = [ctypes.c_void_p]
    L.ra_free.argtypes = [ctypes.c_void_p]
    return L


def first_fit(occ, n):
    run = 0
    for i, used in enumerate(occ):
        run = 0 if used else run + 1
        if run == n:
            return i - n + 1
    return -1


@pytest.mark.parametrize("seed", range(4))
def test_random_admissions_and_releases_match_the_model(ra, seed):
    rng = np.random.default_rng(seed)
    cap = 500
    a = ra.ra_new(cap)
    occ = np.zeros(cap, dtype=bool)
    live = []
    for _ in range(3000):
        if live and rng.random() < 0.45:
            off, n = live.pop(int(rng.integers(len(live))))
            ra.ra_release(a, off, n)
            occ[off:off + n] = False
        elif rng.random() < 0.01:
            cap += int(rng.integers(1, 64))
            ra.ra_grow(a, cap)
            occ = np.concatenate([occ, np.zeros(cap - len(occ), dtype=bool)])
        else:
            n = int(rng.integers(1, 40))
            want = first_fit(occ, n)
            got = ra.ra_alloc(a, n)
            assert got == want
            if got >= 0:
                assert not occ[got:got + n].any()
                occ[got:got + n] = True
                live.append((got, n))
        assert ra.ra_capacity(a) == cap
        used = np.nonzero(occ)[0]
        assert ra.ra_used_end(a) == (int(used[-1]) + 1 if len(used) else 0)
        runs, run = [], 0
        for u in occ:
            run = 0 if u else run + 1
            runs.append(run)
        assert ra.ra_largest_free(a) == (max(runs) if runs else 0)
    ra.ra_free(a)


def test_alloc_at_takes_a_given_free_range_back(ra):
    """alloc_at claims [off, off + len) only when it lies inside one free range, splitting that
    range; a range just released comes back at its own offset even when first fit would not."""
    a = ra.ra_new(100)
    assert ra.ra_alloc(a, 10) == 0
    assert ra.ra_alloc(a, 30) == 10
    ra.ra_release(a, 0, 10)        # free: [0, 10) and [40, 100)
    ra.ra_release(a, 10, 30)       # coalesced: [0, 100)
    assert ra.ra_alloc_at(a, 10, 30) == 1
    assert ra.ra_alloc_at(a, 35, 10) == 0   # overlaps the taken range
    assert ra.ra_alloc(a, 10) == 0          # the left remainder [0, 10)
    assert ra.ra_alloc(a, 60) == 40         # the right remainder [40, 100)
    assert ra.ra_largest_free(a) == 0
    assert ra.ra_alloc_at(a, 99, 2) == 0    # past the capacity
    ra.ra_free(a)
