"""The broadphase's classification of bodies by radius (avbd_broadphase_radii, host code) by the
reference's procedure (tests/radii.test.ts): selection must reproduce the sort-based rule exactly,
and the large-body threshold sits midway to the next radius up (gpu/solver.ts:1268-1272). No GPU."""

import ctypes

import numpy as np

import avbd_b200
from avbd_b200 import _abi

LARGE_FACTOR, MAX_LARGE = 2, 64


def _mulberry32(seed):
    """radii.test.ts:17-25, in 32-bit unsigned arithmetic."""
    s = [seed & 0xFFFFFFFF]
    M = 0xFFFFFFFF

    def imul(a, b):
        return (a * b) & M

    def rnd():
        s[0] = (s[0] + 0x6D2B79F5) & M
        t = s[0]
        t = imul(t ^ (t >> 15), 1 | t)
        t = ((t + imul(t ^ (t >> 7), 61 | t)) & M) ^ t
        return ((t ^ (t >> 14)) & M) / 4294967296
    return rnd


def _by_sort(radii):
    """radii.test.ts:6-14: the classification by sorting."""
    r = sorted(radii)
    n = len(r)
    median = r[n >> 1] if n else 1.0
    small = max([x for x in r if x <= LARGE_FACTOR * median], default=0.0)
    if n > MAX_LARGE:
        small = max(small, r[n - MAX_LARGE - 1])
    return small


def _classify(radii):
    lib = avbd_b200.load()
    a = np.ascontiguousarray(radii, dtype=np.float64)
    small, thr = ctypes.c_double(), ctypes.c_double()
    dp = ctypes.POINTER(ctypes.c_double)
    assert lib.avbd_broadphase_radii(a.ctypes.data_as(dp), len(a), ctypes.byref(small), ctypes.byref(thr)) == _abi.AVBD_OK
    return small.value, thr.value


def test_largest_small_matches_the_sort_based_rule():
    rand = _mulberry32(2)
    cases = [
        [],
        [0.5],
        [0.2165] * 5000 + [2000.0] + [1 + rand() * 6 for _ in range(40)],  # a city of voxels, a ground, a few sections
        [0.2165] * 3000 + [1 + rand() * 6 for _ in range(90)],             # past MAX_LARGE large bodies
        [0.1 + rand() for _ in range(40)],                                 # fewer bodies than MAX_LARGE
        [0.05 + rand() * rand() * 3 for _ in range(20000)],
    ]
    for i, radii in enumerate(cases):
        small, thr = _classify(radii)
        assert small == _by_sort(radii), f'case {i}'
        larger = [x for x in radii if x > small]
        assert thr == (small * 1.5 if not larger else (small + min(larger)) / 2), f'case {i}'


def test_selection_on_runs_of_equal_values():
    """radii.test.ts:27-34's concern: runs of equal values (the median of integers 0..4)."""
    rand = _mulberry32(1)
    for n in (1, 2, 3, 10, 257):
        values = [float(int(rand() * 5)) for _ in range(n)]
        assert _classify(values)[0] == _by_sort(values), n


def test_invalid_radii_are_refused():
    lib = avbd_b200.load()
    dp = ctypes.POINTER(ctypes.c_double)
    for bad in ([1.0, -0.5], [float('nan')]):
        a = np.array(bad)
        assert lib.avbd_broadphase_radii(a.ctypes.data_as(dp), len(a), None, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_broadphase_radii(None, 1, None, None) == _abi.AVBD_ERR_INVALID
