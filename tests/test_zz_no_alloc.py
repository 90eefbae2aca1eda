"""avbd_find_pairs_noalloc (the step's broadphase with every intermediate array in one fixed device
array) against the world's own broadphase: the pair list a world's step finds for the same bodies
(avbd_step, then avbd_read_pairs). Collected last; passes alone in a fresh process too."""

import ctypes

import numpy as np
import pytest

import avbd_b200
from avbd_b200 import CudaSolver3D, _abi, find_pairs_noalloc, scene_records
from avbd_b200._abi import ptr, uptr
from avbd_b200.scenes import Scene, drop_pile, small_world

pytestmark = pytest.mark.gpu


def _as_set(pairs: np.ndarray) -> set:
    return {(int(a), int(b)) for a, b in pairs}


def _world_pairs(scene, groups_mask=None) -> set:
    w = CudaSolver3D(scene)  # creation order: the same indices as the records
    if groups_mask is not None:
        w.set_filters(0, groups_mask)
    w.step(1)
    pairs = w.read_pairs()
    assert w.read_counters()['overflow'] == 0
    w.destroy()
    return _as_set(pairs)


def _cases():
    dense = drop_pile(3000, seed=2, spacing=1.0, layers=3)  # overlapping lattice: thousands of pairs, a large ground
    mixed = small_world(np.random.default_rng(5), 400)  # boxes and spheres, pressed together: every body touches several
    for b in mixed.bodies[1:]:
        b.pos = [b.pos[0] * 0.55, b.pos[1] * 0.55, b.pos[2] * 0.55]
    rng = np.random.default_rng(5)
    groups = rng.integers(1, 4, size=len(mixed.bodies)).astype(np.uint32)
    masks = np.where(rng.uniform(size=len(mixed.bodies)) < 0.3, 0xFFFFFFFE, 0xFFFFFFFF).astype(np.uint32)
    gm = np.stack([groups, masks], axis=1)
    return [(dense, None), (mixed, gm)]


def test_noalloc_pairs_match_world_broadphase(cuda_lib):
    cases = _cases()
    # two calls in a row on different bodies, then the first again: the shared array is reset per call
    got = [find_pairs_noalloc(scene_records(s)[0], gm) for s, gm in cases]
    got.append(find_pairs_noalloc(scene_records(cases[0][0])[0], cases[0][1]))
    want = [_world_pairs(s, gm) for s, gm in cases]
    for g, wset, (s, _) in zip(got, want + [want[0]], cases + [cases[0]]):
        assert np.all(g[:, 0] > g[:, 1]), s.name
        assert len(g) == len(_as_set(g)), f'{s.name}: a pair found twice'
        assert _as_set(g) == wset, f'{s.name}: {len(_as_set(g) - wset)} extra, {len(wset - _as_set(g))} missing of {len(wset)}'
    assert len(want[0]) > 2000 and len(want[1]) > 100


def test_noalloc_rejects_past_its_limits(cuda_lib):
    big = drop_pile(avbd_b200._abi.NOALLOC_MAX_BODIES + 1, seed=3, spacing=2.0, layers=4)
    with pytest.raises(avbd_b200.AvbdError, match='at most 4096'):
        find_pairs_noalloc(scene_records(big)[0])
    dense, _ = _cases()[0]
    with pytest.raises(avbd_b200.AvbdError, match='more than the 10'):
        find_pairs_noalloc(scene_records(dense)[0], cap=10)
    # and the next call is whole again
    assert _as_set(find_pairs_noalloc(scene_records(dense)[0])) == _world_pairs(dense)


def _sphere_lattice(side: int = 16, spacing: float = 0.6, r: float = 0.61) -> Scene:
    """side^3 spheres whose neighbours up to two lattice steps away overlap: 57372 pairs at 16^3."""
    s = Scene('sphere lattice')
    for i in range(side):
        for j in range(side):
            for k in range(side):
                s.sphere(r, 1, 0.5, [i * spacing, j * spacing, 5 + k * spacing])
    return s


def _call(lib, bodies, gm, cap):
    out = np.zeros(2 * max(cap, 1), dtype=np.uint32)
    count = ctypes.c_uint32(12345)
    code = lib.avbd_find_pairs_noalloc(ptr(bodies), len(bodies), uptr(gm) if gm is not None else None, uptr(out), cap, ctypes.byref(count), None)
    return code, count.value, out


def test_noalloc_c_limits(cuda_lib):
    """The C entry point's own refusals, called directly (the Python guard bypassed): past the body
    maximum (*count 0), past the pair maximum with a larger cap (*count = every pair found), and a
    hull shape code (no hull buffer to read it against)."""
    lib = cuda_lib
    big = scene_records(drop_pile(_abi.NOALLOC_MAX_BODIES + 1, seed=3, spacing=2.0, layers=4))[0]
    code, count, _ = _call(lib, big, None, 1024)
    assert code == _abi.AVBD_ERR_CAPACITY and count == 0
    lattice = _sphere_lattice()
    recs = scene_records(lattice)[0]
    assert len(recs) == _abi.NOALLOC_MAX_BODIES
    code, count, out = _call(lib, recs, None, 65536)
    want = _world_pairs(lattice)
    assert code == _abi.AVBD_ERR_CAPACITY and count == len(want) > _abi.NOALLOC_MAX_PAIRS
    kept = _as_set(out[:2 * _abi.NOALLOC_MAX_PAIRS].reshape(-1, 2))
    assert len(kept) == _abi.NOALLOC_MAX_PAIRS and kept <= want  # the pairs that fit are real ones
    hull = recs[:8].copy()
    hull['shape'][3] = 3.0
    code, count, _ = _call(lib, hull, None, 1024)
    assert code == _abi.AVBD_ERR_INVALID and count == 0
    with pytest.raises(avbd_b200.AvbdError, match='groups_mask holds'):
        find_pairs_noalloc(recs[:8], np.ones(8, dtype=np.uint32))
    # and a whole call afterwards
    dense, _ = _cases()[0]
    assert _as_set(find_pairs_noalloc(scene_records(dense)[0])) == _world_pairs(dense)
