"""The passes a World runs around the step, through the C ABI, against their CPU restatement
(oracle/queries.py) on the same f32 records: impulses on bodies (Pusher, src/lib/push.ts), contact
begin/end events (ContactWatch, src/lib/contacts.ts) and nearest-hit raycasts (Raycaster,
src/lib/raycast.ts)."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200 import _abi
from avbd_b200.scenes import Scene, drop_pile, hull_pile
import queries

pytestmark = pytest.mark.gpu


def test_pushes_match_oracle(cuda_lib):
    scene = drop_pile(400, seed=3, spacing=1.6, layers=3)
    w = avbd_b200.CudaSolver3D(scene)
    w.step(20)
    w.set_lifecycle(7, 2)  # disabled: left alone
    before = w.read_bodies()
    rng = np.random.default_rng(1)
    others = np.setdiff1d(np.arange(len(before)), [0, 7])
    # the static ground and the disabled body are left alone; 58 others are pushed
    slots = np.concatenate([[0, 7], rng.choice(others, size=58, replace=False)])
    p = np.zeros(len(slots), dtype=_abi.PUSH_DTYPE)
    p['body'] = slots
    p['lin'] = rng.normal(0, 5, (len(slots), 3))
    p['off_lin'] = p['lin'] * rng.uniform(0, 1, (len(slots), 1))
    at = before['pos'][slots] + rng.normal(0, 0.3, (len(slots), 3))
    p['moment'] = np.cross(at, p['off_lin']) + rng.normal(0, 0.5, (len(slots), 3))
    w.apply_pushes(p)
    after = w.read_bodies()
    vel, avel = queries.apply_pushes(before, p)
    assert np.allclose(after['vel'], vel, rtol=1e-5, atol=1e-5) and np.allclose(after['ang_vel'], avel, rtol=1e-5, atol=1e-4)
    assert np.array_equal(after['vel'][[0, 7]], before['vel'][[0, 7]])
    moved = np.abs(after['vel'] - before['vel']).max(axis=1) > 0
    assert moved.sum() == len(slots) - 2
    for bad in (np.r_[p[:2], p[:1]], p[:1].copy()):
        if len(bad) == 1:
            bad['body'] = len(before)  # not a slot
        with pytest.raises(avbd_b200.AvbdError):
            w.apply_pushes(bad)
    w.destroy()


def _bouncing_boxes():
    s = Scene('boxes dropped and kicked')
    s.box([40, 40, 1], 0, 0.5, [0, 0, -0.5])
    for k in range(24):
        s.box([0.6, 0.6, 0.6], 1, 0.5, [(k % 6) * 1.5 - 4, (k // 6) * 1.5 - 2, 0.8 + 0.4 * (k % 3)])
    return s


def test_contact_events_match_oracle(cuda_lib):
    """24 boxes land (begins), some are kicked up off the ground (ends) and land again (begins); half
    of them report. Every event, its step, point, impulse and normal against the restatement run on
    the same contacts read back after each step."""
    s = _bouncing_boxes()
    w = avbd_b200.CudaSolver3D(s)
    n = len(s.bodies)
    watch = w.contact_watch(pairs=256, capacity=4096)
    ids = np.arange(n) + 100
    on = (np.arange(n) % 2 == 1)
    on[0] = False  # the ground does not report; its pairs with reporting boxes do
    watch.set_watched(np.arange(n), ids, on)
    model = {i: (int(ids[i]), bool(on[i])) for i in range(n)}
    dt = s.params.dt
    prev, want = set(), []
    for step in range(1, 121):
        if step == 50:  # the reporting boxes kicked up at 4 m/s: they leave the ground and land again
            b = w.read_bodies()
            kick = np.zeros(12, dtype=_abi.PUSH_DTYPE)
            kick['body'] = np.arange(1, 25, 2)
            kick['lin'][:, 2] = 4.0 * b['mass'][kick['body']]
            w.apply_pushes(kick)
        w.step()
        watch.run(step, dt)
        m, c = w.read_contacts()
        events, prev = queries.contact_events(prev, m, c, w.read_bodies(), model, step, dt)
        want += events
    got, dropped, full = watch.read()
    assert dropped == 0 and not full
    kinds = {k: sum(1 for e in want if e[0] == k) for k in (1, 2)}
    assert kinds[1] >= 20 and kinds[2] >= 10, kinds
    key = lambda e: (e[3], e[0], e[1], e[2])
    want.sort(key=key)
    got_l = sorted(got.tolist(), key=lambda e: (e[3], e[0], e[1], e[2]))
    assert [key(e) for e in want] == [(e[3], e[0], e[1], e[2]) for e in got_l]
    for wv, g in zip(want, got_l):
        if wv[0] == 1:
            assert np.allclose(g[4], wv[4], atol=1e-5) and abs(g[5] - wv[5]) <= 1e-5 * max(1.0, wv[5]) and np.allclose(g[6], wv[6], atol=1e-6)
    assert np.all(np.diff(got['step'].astype(np.int64)) >= 0)  # read gives step order
    # a capacity too small drops the rest and says how many
    small = w.contact_watch(pairs=256, capacity=2)
    small.set_watched(np.arange(n), ids, np.ones(n, bool))
    w.step()
    small.run(121, dt)
    ev, dropped, _ = small.read()
    assert len(ev) == 2 and dropped > 0
    small.destroy()
    watch.destroy()
    w.destroy()


def test_raycast_matches_oracle(cuda_lib):
    """Rays among hulls, boxes and spheres: the nearest body (the lowest slot on a tie), its distance
    and the world normal there; rays from inside a body; a distance cap; ignored slots and a group mask."""
    s = hull_pile(90, seed=4)
    w = avbd_b200.CudaSolver3D(s)
    w.step(40)
    bodies = w.read_bodies()
    rng = np.random.default_rng(7)
    n = 300
    origins = rng.uniform(-6, 6, (n, 3)) + np.array([0, 0, 3.0])
    origins[:20] = bodies['pos'][1:21]  # inside bodies: distance 0
    directions = rng.normal(0, 1, (n, 3))
    maxd = np.where(rng.uniform(size=n) < 0.2, rng.uniform(0.5, 3, n), 3.0e38).astype(np.float32)
    groups = np.ones(len(bodies), np.uint32)
    groups[5:15] = 2
    w.set_filters(0, np.stack([groups, np.full(len(bodies), 0xFFFFFFFF, np.uint32)], axis=1))
    filters = np.stack([groups, groups], axis=1)
    ignore = [3, 30, 31]
    for mask in (0xFFFFFFFF, 1):
        hits = w.raycast(origins, directions, maxd, ignore=ignore, mask=mask)
        rays = np.zeros(n, _abi.RAY_DTYPE)  # the f32 inputs the device traced
        rays['origin'], rays['direction'], rays['max_distance'] = origins, directions, maxd
        agree = 0
        for k in range(n):
            d = rays['direction'][k].astype(float)
            d = (d / np.linalg.norm(d)).astype(np.float32)
            want = queries.raycast(bodies, s.hull_words, filters, rays['origin'][k], d, float(rays['max_distance'][k]), ignore=ignore, mask=mask)
            h = hits[k]
            if want is None:
                assert h['body'] == -1, f'ray {k}: hit {h["body"]}, none expected'
                continue
            b, t, nrm = want
            assert h['body'] >= 0, f'ray {k}: no hit, body {b} expected'
            assert abs(h['distance'] - t) <= 1e-5 * max(1.0, t), f'ray {k}: distance {h["distance"]} vs {t}'
            if h['body'] == b:
                if not np.allclose(h['normal'], nrm, atol=1e-4):  # faces that tie, or a grazing ray on a sphere
                    ties = queries.normals_at(bodies[b], s.hull_words, rays['origin'][k], d, float(h['distance']), 1e-5 * max(1.0, t))
                    assert any(np.allclose(h['normal'], m, atol=1e-4) for m in ties), f'ray {k}: normal {h["normal"]} vs {nrm}'
                agree += 1
            else:  # only where two surfaces lie at the same distance
                other = queries.ray_trace(bodies[h['body']], s.hull_words, rays['origin'][k], d, float(rays['max_distance'][k]))
                assert other is not None and abs(other[0] - t) <= 1e-5 * max(1.0, t)
            assert h['body'] not in ignore and (groups[h['body']] & mask)
        assert agree > n // 4
    with pytest.raises(avbd_b200.AvbdError):
        w.raycast(origins[:1], directions[:1], ignore=list(range(17)))
    w.destroy()


def test_pose_capture_frames_match_the_world_and_round_trip(cuda_lib):
    """Pose cache frames gathered on the device every 3 steps of a pile equal the poses read back at
    those steps bit for bit, stamped with the world's step word; frames past max_frames are dropped and
    counted; the capture encodes to the pose cache format (src/bake/pose-cache.ts) and decodes to the
    same frames."""
    from avbd_b200 import pose_cache as pc
    from avbd_b200.scenes import drop_pile
    w = avbd_b200.CudaSolver3D(drop_pile(500, seed=2))
    cap = w.pose_capture(max_frames=5)
    seen, words = [], []
    for _ in range(6):
        w.step(3)
        cap.frame()
        b = w.read_bodies()
        seen.append(np.concatenate([b['pos'], b['rot']], axis=1).astype(np.float32))
        words.append(w.read_counters()['steps'])
    steps, poses, dropped = cap.read()
    assert len(steps) == 5 and dropped == 1
    assert list(steps) == words[:5]
    assert np.array_equal(poses.view(np.uint32), np.stack(seen[:5]).view(np.uint32))
    cache = cap.to_pose_cache(77, provenance={'tool': 'test'})
    manifest, chunks = pc.encode_pose_cache(cache, frames_per_chunk=2)
    back = pc.decode_pose_cache(manifest, chunks)
    assert np.array_equal(back.poses.view(np.uint32), poses.view(np.uint32)) and np.array_equal(back.steps, steps)
    assert back.bodies[0].fixed and not back.bodies[1].fixed  # the ground is static
    cap.reset()
    cap.frame()
    assert len(cap.read()[0]) == 1
    cap.destroy()
    w.destroy()
