"""Convex hulls on the GPU (the hull narrowphase of src/avbd3d/gpu/wgsl-hull.ts) against the CPU
oracle's f32 restatement and its FP64 GPU-mode step, through the C ABI."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200.scenes import hull_pairs, hull_pile
from oracle import Oracle
from _util import cuda_from_oracle, pose_diff

pytestmark = pytest.mark.gpu


def test_hull_narrowphase_known_answers(cuda_lib):
    """As avbd3d-gpu.gpu.test.ts:101-142 for hulls: 200 overlapping pairs of a hull with a hull, a
    box or a sphere; feature keys and anchors bit for bit the oracle's f32 restatement, and the FP64
    narrowphase's points within 1e-3 where it picks the same features."""
    s = hull_pairs(200, seed=5)
    w = avbd_b200.CudaSolver3D(s)
    w.step()
    c = w.read_counters()
    assert c['error'] == 0 and c['overflow'] == 0
    contacts = w.read_contact_list()
    o32, o64 = Oracle(s, fp32=True), Oracle(s)
    total = same64 = pairs64 = 0
    kinds = {}
    for p in range(200):
        a, b = 2 * p + 1, 2 * p
        mine = [x for x in contacts if x['a'] == a and x['b'] == b]
        exact, _ = o32.narrowphase(a, b)
        assert len(mine) == len(exact), f'pair {p}: {len(mine)} contacts vs {len(exact)}'
        total += len(exact)
        for x, (f, ra, rb) in zip(mine, exact):
            assert x['feature'] == f, f'pair {p}: feature {x["feature"]:#x} vs {f:#x}'
            assert np.array_equal(x['rA'].astype(np.float32), ra.astype(np.float32)), f'pair {p}: rA {x["rA"]} vs {ra}'
            assert np.array_equal(x['rB'].astype(np.float32), rb.astype(np.float32)), f'pair {p}: rB'
            kinds[f >> 24] = kinds.get(f >> 24, 0) + 1
        ref, _ = o64.narrowphase(a, b)
        if [f for f, _, _ in ref] == [f for f, _, _ in exact]:
            pairs64 += 1
            for (f, ra, rb), (_, ra32, rb32) in zip(ref, exact):
                assert np.linalg.norm(ra - ra32) < 1e-3 and np.linalg.norm(rb - rb32) < 1e-3
                same64 += 1
    print(f'hull narrowphase: {total} contacts, feature kinds {kinds}; FP64 picks the same features on {pairs64} of 200 pairs')
    assert total > 200 and len(contacts) == total
    assert kinds.get(0, 0) + kinds.get(1, 0) > 0 and kinds.get(3, 0) > 0  # face and sphere contacts seen
    assert pairs64 >= 190


def test_hull_pile_coloured_step_matches_fp64(cuda_lib):
    """A pile of hulls, boxes and spheres (coloured mode): from the oracle's state after 70 GPU-mode
    steps, one GPU step against one FP64 step with the oracle's colours; poses within 1e-5."""
    s = hull_pile(300, seed=7)
    o = Oracle(s)
    for _ in range(70):
        o.step_gpu()
    man, _ = o.manifolds()
    assert len(man) > 200
    w = cuda_from_oracle(o, s.params, hulls_from=s)
    o.step_gpu()
    w.set_fixed_colors(o.colors())
    w.step()
    c = w.read_counters()
    assert c['error'] == 0 and c['overflow'] == 0
    d = pose_diff(w.read_bodies(), o.bodies())
    print(f'hull pile coloured step: pose diff {d:.3e}, {len(man)} manifolds')
    assert d < 1e-5
    w.destroy()


def test_hull_pile_settles_deterministically(cuda_lib):
    """2000 hulls (with boxes and spheres) dropped and settled: the same bits twice, nothing through
    the ground, no error or overflow."""
    s = hull_pile(2000, seed=8)
    runs = []
    for _ in range(2):
        w = avbd_b200.CudaSolver3D(s, spatial_sort=True)
        w.step(150)
        c = w.read_counters()
        assert c['error'] == 0 and c['overflow'] == 0 and c['manifolds'] > 1000
        b = w.read_bodies()
        moving = b['mass'] > 0
        assert np.isfinite(b['pos']).all() and b['pos'][moving, 2].min() > -0.2
        runs.append(b.view(np.uint32).copy())
        w.destroy()
    assert np.array_equal(runs[0], runs[1])


def test_hull_records_are_validated(cuda_lib):
    s = hull_pile(10, seed=1)
    w = avbd_b200.CudaSolver3D(body_capacity=64)
    rec = s.hull_words[:4 * (s.hull_offsets[1] if len(s.hull_offsets) > 1 else len(s.hull_words) // 4)].copy()
    bad = rec.copy()
    bad[1] = 40  # more vertices than a hull may have
    with pytest.raises(avbd_b200.AvbdError):
        w.add_hull(bad)
    at = w.add_hull(rec)
    body = avbd_b200.pack_bodies([s.bodies[1]])
    body['shape'] = 3 + at + 1  # not a hull header
    with pytest.raises(avbd_b200.AvbdError):
        w.add_bodies(body)
    body['shape'] = 3 + at
    w.add_bodies(body)
    w.destroy()


def test_hull_release_and_reuse(cuda_lib):
    """releaseHull / unpinHull (gpu/solver.ts:1408-1454): a released record's run is reused by the
    next hull that fits; a record a body names is not released; bodies keep colliding."""
    s = hull_pile(10, seed=1)
    offs = list(s.hull_offsets) + [len(s.hull_words) // 4]
    recs = [s.hull_words[4 * offs[k]:4 * offs[k + 1]].copy() for k in range(len(offs) - 1)]
    for r, o in zip(recs, offs):
        r[[0, 2, 4, 6]] -= np.uint32(o)  # each record with its header at vec4 0
    big = max(range(len(recs)), key=lambda k: len(recs[k]))
    small = min(range(len(recs)), key=lambda k: len(recs[k]))
    w = avbd_b200.CudaSolver3D(body_capacity=64)
    a = w.add_hull(recs[big])
    b = w.add_hull(recs[small])
    body = avbd_b200.pack_bodies([s.bodies[1]])
    body['shape'] = 3 + b
    w.add_bodies(body)
    with pytest.raises(avbd_b200.AvbdError):
        w.release_hull(b)  # a body names it
    w.release_hull(a)
    st = w.hull_storage()
    assert st['largest_free'] == len(recs[big]) // 4
    c = w.add_hull(recs[small])
    assert c == a  # first fit: the released run
    assert w.hull_storage()['largest_free'] == (len(recs[big]) - len(recs[small])) // 4
    body['shape'] = 3 + c
    w.add_bodies(body)
    w.step(5)
    assert w.read_counters()['error'] == 0
    with pytest.raises(avbd_b200.AvbdError):
        w.release_hull(a + 1)  # not a record
    w.destroy()
