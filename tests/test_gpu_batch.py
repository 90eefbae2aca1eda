"""Batched worlds (avbd_batch_*) against the single-world step and the CPU oracle, per world."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200 import BatchSolver3D, CudaSolver3D
from avbd_b200.scenes import batched_worlds, cube_pyramid, demo_scene, drop_pile
from oracle import Oracle
from _util import cuda_from_oracle, oracle_sequential_colors, pose_diff

pytestmark = pytest.mark.gpu

JOINT_SCENES = ['Rope', 'Heavy Rope', 'Spring', 'Bridge', 'Breakable', 'Soft Body', 'Stack']


def _mixed_scenes():
    """Small generated worlds of every size class plus the demo scenes with joints and springs."""
    scenes = batched_worlds(10, seed=11)
    scenes += [demo_scene(n) for n in JOINT_SCENES]
    scenes.append(cube_pyramid(8))
    for s in scenes:  # a batch's worlds share one parameter set
        s.params = scenes[0].params
    return scenes


def _batch_for(scenes, **kw):
    n = sum(len(s.bodies) for s in scenes)
    nj = sum(sum(1 for f in s.forces if f.kind != 'ignore') for s in scenes)
    b = BatchSolver3D(len(scenes), n, nj, params=scenes[0].params, **kw)
    for s in scenes:
        b.add_scene(s)
    return b


def _pose_gap(a, b):
    return max(float(np.abs(a['pos'] - b['pos']).max()), float(np.abs(a['rot'] - b['rot']).max()))


def test_batch_world_matches_single_world(cuda_lib):
    """Every world of a batch steps as the same scene does alone. Against a single world whose
    solve runs as one block (the batch's scope) the batch is bit-identical over 30 steps: pairs,
    colours, joints and poses. Against the default full-grid launch (whose lane groups sum a body's
    rows in another order) poses agree within 1e-5 after one step."""
    scenes = _mixed_scenes()
    b = _batch_for(scenes)
    singles = [CudaSolver3D(s) for s in scenes]
    grid = [CudaSolver3D(s) for s in scenes]
    for w in singles:
        w.set_solve_blocks(1)
    b.step(1)
    for w in singles + grid:
        w.step(1)
    b.synchronize()
    for i, (w, g) in enumerate(zip(singles, grid)):
        got = b.read_bodies(i)
        gap = _pose_gap(got, g.read_bodies())
        assert gap < 1e-5, f'{scenes[i].name}: pose gap {gap} to the full-grid step'
        cb, cw = b.read_counters(i), g.read_counters()
        assert cb['error'] == 0 and cb['overflow'] == 0, scenes[i].name
        assert (cb['pairs'], cb['contacts'], cb['colors']) == (cw['pairs'], cw['contacts'], cw['colors']), scenes[i].name
        assert np.array_equal(b.read_colors(i), g.read_colors()), scenes[i].name
        g.destroy()
    b.step(29)
    for w in singles:
        w.step(29)
    b.synchronize()
    for i, w in enumerate(singles):
        got, want = b.read_bodies(i), w.read_bodies()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f'{scenes[i].name}: pose gap {_pose_gap(got, want)} after 30 steps'
        assert np.array_equal(b.read_colors(i), w.read_colors()), scenes[i].name
        jb, ib = b.read_joints(i)
        jw, iw = w.read_joints()
        assert np.array_equal(jb.view(np.uint32), jw.view(np.uint32)) and np.array_equal(ib, iw), f'{scenes[i].name}: joints differ'
        cb, cw = b.read_counters(i), w.read_counters()
        assert (cb['pairs'], cb['contacts'], cb['manifolds']) == (cw['pairs'], cw['contacts'], cw['manifolds']), scenes[i].name
        w.destroy()
    b.destroy()


def test_batch_seeded_step_matches_oracle(cuda_lib):
    """avbd3d-gpu.gpu.test.ts:35-99 per world of a batch: the oracle's state seeded into single
    worlds, those continued as batch worlds (add_world_from), one batch step against one FP64
    oracle step with the same colours. Poses within 1e-5 where no feature key tied; the 8-row
    pyramid in coloured mode (GPU-mode oracle)."""
    names = ['Ground', 'Static Friction', 'Rope', 'Heavy Rope', 'Spring', 'Spring Ratio', 'Stack', 'Stack Ratio', 'Breakable']
    oracles, seeded = [], []
    for name in names:
        scene = demo_scene(name)
        o = Oracle(scene)
        o.step(60)
        w = cuda_from_oracle(o, scene.params)
        w.set_fixed_colors(oracle_sequential_colors(o))
        oracles.append((name, o, False))
        seeded.append(w)
    pyr = cube_pyramid(8, gravity=-10.0)
    o = Oracle(pyr)
    for _ in range(40):
        o.step_gpu()
    w = cuda_from_oracle(o, pyr.params)
    o.step_gpu()  # the oracle's own colours for this step
    w.set_fixed_colors(o.colors())
    oracles.append(('pyramid 8', o, True))
    seeded.append(w)
    b = BatchSolver3D(len(seeded), sum(x.body_count for x in seeded), 256, params=demo_scene('Stack').params)
    for w in seeded:
        b.add_world_from(w)
    b.step()
    b.synchronize()
    worst = 0.0
    for i, (name, o, gpu_mode) in enumerate(oracles):
        if not gpu_mode:
            o.step()
        c = b.read_counters(i)
        assert c['error'] == 0 and c['overflow'] == 0, name
        d = pose_diff(b.read_bodies(i), o.bodies())
        worst = max(worst, d)
        assert d < 1e-5, f'{name}: pose diff {d}'
    print(f'batch seeded step vs oracle: worst pose diff {worst:.3e}')
    for w in seeded:
        w.destroy()
    b.destroy()


def test_batch_pair_storage_grows_per_world(cuda_lib):
    """Worlds whose pair slots run short are laid out again with more (the single world's adapt rule);
    the batch ends as one that had room from the start."""
    scenes = batched_worlds(6, seed=5, median=200)
    small = _batch_for(scenes, pairs_per_body=1)
    ample = _batch_for(scenes, pairs_per_body=8)
    overflowed = False
    for _ in range(60):
        for b in (small, ample):
            b.step()
            b.synchronize()
        overflowed |= any(small.read_counters(i)['overflow'] for i in range(len(scenes)))
    assert small.info()['relayouts'] > 0
    for i in range(len(scenes)):
        assert small.read_counters(i)['overflow'] == 0
        assert small.world_info(i)['pair_capacity'] > ample.world_info(i)['pair_capacity'] // 8
        if not overflowed:
            assert np.array_equal(small.read_bodies(i).view(np.uint32), ample.read_bodies(i).view(np.uint32))
        assert np.isfinite(small.read_bodies(i)['pos']).all()
    small.destroy()
    ample.destroy()


def test_batch_graphs_and_determinism(cuda_lib):
    """A batch replayed from CUDA graphs ends in the same bits as direct launches, run after run."""
    scenes = batched_worlds(40, seed=8)
    out = []
    for graphs in (True, False, True):
        b = _batch_for(scenes)
        b.use_graphs(graphs)
        b.step(40)
        b.synchronize()
        assert b.info()['graphs'] == (1 if graphs else 0)
        out.append(np.concatenate([b.read_bodies(i) for i in range(len(scenes))]).view(np.uint32).copy())
        b.destroy()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


def test_batch_sub_block_worlds_match_block_per_world(cuda_lib):
    """Four warps, two warps or one warp a world (two, four or eight worlds a block, named barriers or
    warp barriers between colour passes) step every world bit for bit as a block a world does, over
    30 steps of joints, springs, stacks and piles, with one row a lane and with four; the shape is
    reported back and bad shapes are refused."""
    scenes = _mixed_scenes()
    for rpl in (1, 4):
        out = []
        for wt in (256, 128, 64, 32):
            b = _batch_for(scenes)
            b.set_launch(collide_threads=128, solve_blocks=0, rows_per_lane=rpl, world_threads=wt)
            info = b.info()
            assert (info['world_threads'], info['rows_per_lane']) == (wt, rpl)
            b.step(30)
            b.synchronize()
            for i in range(len(scenes)):
                c = b.read_counters(i)
                assert c['error'] == 0 and c['overflow'] == 0, scenes[i].name
            bodies = np.concatenate([b.read_bodies(i) for i in range(len(scenes))]).view(np.uint32).copy()
            joints = np.concatenate([b.read_joints(i)[0] for i in range(len(scenes))]).view(np.uint32).copy()
            colors = np.concatenate([b.read_colors(i) for i in range(len(scenes))]).copy()
            out.append((bodies, joints, colors))
            b.destroy()
        b0, j0, c0 = out[0]
        for wt, (b1, j1, c1) in zip((128, 64, 32), out[1:]):
            assert np.array_equal(c0, c1), f'{wt} threads a world, rows a lane {rpl}: colours differ'
            assert np.array_equal(j0, j1), f'{wt} threads a world, rows a lane {rpl}: joints differ'
            assert np.array_equal(b0, b1), f'{wt} threads a world, rows a lane {rpl}: bodies differ'
    b = _batch_for(scenes[:2])
    for bad in ((100, 0, 1, 256), (128, 0, 0, 256), (128, 0, 1, 96), (128, 10 ** 6, 1, 32)):
        with pytest.raises(avbd_b200.AvbdError):
            b.set_launch(*bad)
    b.destroy()


def test_batch_tuner_and_host_buffers(cuda_lib):
    """The autotuner times each launch shape and keeps the fastest; all bodies round-trip through
    host buffers on the batch's stream."""
    scenes = batched_worlds(64, seed=9)
    b = _batch_for(scenes)
    b.step(5)
    t = b.tune(2)
    assert len(t['candidates']) >= 6 and all(c['ms_per_step'] > 0 for c in t['candidates'])
    assert {c['rows_per_lane'] for c in t['candidates']} == {1, 4} and t['rows_per_lane'] in (1, 4)  # bodies per warp tuned too
    assert {c['world_threads'] for c in t['candidates']} == {32, 64, 128, 256} and t['world_threads'] in (32, 64, 128, 256)  # threads a world
    assert t['ms_per_step'] == min(c['ms_per_step'] for c in t['candidates'])
    info = b.info()
    assert info['collide_threads'] == t['collide_threads'] and info['solve_blocks'] == t['solve_blocks']
    assert info['world_threads'] == t['world_threads'] and info['rows_per_lane'] == t['rows_per_lane']
    n = info['bodies']
    host = np.zeros(n, dtype=avbd_b200.BODY_DTYPE)
    b.read_all_bodies_into(host)
    for i in range(len(scenes)):
        wi = b.world_info(i)
        assert np.array_equal(host[wi['first_body']:wi['first_body'] + wi['bodies']].view(np.uint32), b.read_bodies(i).view(np.uint32))
    host['vel'] *= 0.5
    b.write_all_bodies_async(host)
    back = np.zeros_like(host)
    b.read_all_bodies_into(back)
    assert np.array_equal(back.view(np.uint32), host.view(np.uint32))
    b.step(3)
    b.synchronize()
    b.destroy()


def test_batch_rejects_bad_worlds(cuda_lib):
    b = BatchSolver3D(2, 64, 4)
    s = drop_pile(80, seed=1, spacing=1.6, layers=2)
    with pytest.raises(avbd_b200.AvbdError):
        b.add_scene(s)  # more bodies than the batch holds
    ok = drop_pile(20, seed=1, spacing=1.6, layers=2)
    b.add_scene(ok)
    bodies, _, _, _ = avbd_b200.scene_records(ok)
    bodies['pos'][3, 0] = np.nan
    with pytest.raises(avbd_b200.AvbdError):
        b.add_world(bodies)
    with pytest.raises(avbd_b200.AvbdError):
        b.read_bodies(5)
    b.step(2)
    b.synchronize()
    b.destroy()
