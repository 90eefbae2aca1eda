"""The CUDA step against the CPU oracle: the reference's own GPU/CPU procedures
(tests-gpu/avbd3d-gpu.gpu.test.ts, tests-gpu/pivot.gpu.test.ts) through the C ABI."""

import math

import numpy as np
import pytest

import avbd_b200
from avbd_b200.scenes import Scene, demo_scene, cube_pyramid, drop_pile
from oracle import NO_COLOR, Oracle, color_graph
from _util import (contact_map, cuda_from_oracle, lambda_parity, lcg, oracle_contact_map, oracle_sequential_colors, pose_diff, qnormalize,
                   params_struct)

pytestmark = pytest.mark.gpu

# Scenes with at most 64 dynamic bodies (one colour each): avbd3d-gpu.gpu.test.ts:31-32
PARITY_SCENES = ['Ground', 'Dynamic Friction', 'Static Friction', 'Rope', 'Heavy Rope', 'Spring', 'Spring Ratio', 'Stack', 'Stack Ratio', 'Breakable']


def test_seeded_single_step_matches_reference(cuda_lib):
    """avbd3d-gpu.gpu.test.ts:35-99: seed the reference's full state (rounded to f32, so both start
    from the same values), one colour per body in its Gauss-Seidel order, one step each; contacts at
    the same points (1e-4), every multiplier row within 1e-5 relative plus the stated floor
    (_util.lambda_parity), poses within 1e-5 where no feature key tied (the reference's own test
    holds lambda to 1e-3, :77)."""
    tie_frames = 0
    worst_pose = worst_lam = worst_ratio = 0.0
    for name in PARITY_SCENES:
        scene = demo_scene(name)
        o = Oracle(scene)
        frame = 0
        for at in (60, 120, 300):
            o.step(at - frame)
            frame = at
            o.round_f32()
            w = cuda_from_oracle(o, scene.params)
            w.set_fixed_colors(oracle_sequential_colors(o))
            w.step()
            o.step()
            frame += 1
            where = f'{name} frame {at}'
            counters = w.read_counters()
            assert counters['overflow'] == 0 and counters['error'] == 0, where
            contacts = w.read_contact_list()
            bodies = w.read_bodies()
            ob = o.bodies()
            man, con = o.manifolds()
            keys_match = True
            expected = 0
            k = 0
            for m in man:
                a, b, cnt = int(m[1]), int(m[2]), int(m[3])
                pts = con[k:k + cnt]
                k += cnt
                if ob[a, 19] <= 0 and ob[b, 19] <= 0:
                    continue
                for q in pts:
                    expected += 1
                    g = [c for c in contacts if c['a'] == a and c['b'] == b and np.linalg.norm(c['rA'] - q[2:5]) < 1e-4 and np.linalg.norm(c['rB'] - q[5:8]) < 1e-4]
                    assert g, f'{where}: contact {a}-{b} at {q[2:5]} not found'
                    g = g[0]
                    if g['feature'] != int(q[0]):
                        keys_match = False
            assert len(contacts) == expected, f'{where}: contact count {len(contacts)} vs {expected}'
            if not keys_match:
                tie_frames += 1
            else:
                lp = lambda_parity(contact_map(*w.read_contacts()), oracle_contact_map(o))
                worst_ratio, worst_lam = max(worst_ratio, lp['ratio']), max(worst_lam, lp['worst_rel'])
                assert lp['ratio'] <= 1.0, f'{where}: lambda {lp}'
                d = pose_diff(bodies, ob)
                worst_pose = max(worst_pose, d)
                assert d < 1e-5, f'{where}: pose diff {d}'
            w.destroy()
    print(f'seeded single step: worst pose diff {worst_pose:.3e}, lambda: worst rel (|lambda| > 1e-3) {worst_lam:.3e}, '
          f'worst |d| / bound {worst_ratio:.2f}, tie frames {tie_frames}')
    # Only Dynamic Friction's flat boxes tie (avbd3d-gpu.gpu.test.ts:96-97)
    assert tie_frames <= 2


def _box_pairs(count=300, seed=7):
    rand = lcg(seed)
    s = Scene('box pairs')
    s.params.gravity = 0.0
    s.params.iterations = 0
    for p in range(count):
        base = [(p % 20) * 20, (p // 20) * 20, 0]
        for k in range(2):
            size = [0.4 + rand() * 1.6, 0.4 + rand() * 1.6, 0.4 + rand() * 1.6]
            off = [0, 0, 0] if k == 0 else [(rand() - 0.5) * 1.2, (rand() - 0.5) * 1.2, (rand() - 0.5) * 1.2]
            i = s.box(size, 1, 0.5, [base[0] + off[0], base[1] + off[1], base[2] + off[2]])
            s.bodies[i].rot = qnormalize([rand() - 0.5, rand() - 0.5, rand() - 0.5, rand() - 0.5])
    return s


def test_narrowphase_known_answers(cuda_lib):
    """avbd3d-gpu.gpu.test.ts:101-142: 300 random overlapping box pairs; the same contacts as the
    f64 reference (1e-3) with the same feature keys, and bit for bit the f32 restatement."""
    s = _box_pairs()
    w = avbd_b200.CudaSolver3D(s)
    w.step()
    contacts = w.read_contact_list()
    o64, o32 = Oracle(s), Oracle(s, fp32=True)
    total = 0
    for p in range(300):
        a, b = 2 * p + 1, 2 * p
        mine = [c for c in contacts if c['a'] == a and c['b'] == b]
        ref, _ = o64.narrowphase(a, b)
        exact, _ = o32.narrowphase(a, b)
        assert len(mine) == len(ref) == len(exact), f'pair {p}: counts {len(mine)} {len(ref)} {len(exact)}'
        total += len(ref)
        for f, ra, rb in ref:
            g = [c for c in mine if np.linalg.norm(c['rA'] - ra) < 1e-3 and np.linalg.norm(c['rB'] - rb) < 1e-3]
            assert g and g[0]['feature'] == f, f'pair {p}: contact at {ra}'
        # bit for bit: same order, keys and f32 anchors
        for c, (f, ra, rb) in zip(mine, exact):
            assert c['feature'] == f
            assert np.array_equal(c['rA'].astype(np.float32), ra.astype(np.float32)), f'pair {p}: rA {c["rA"]} vs {ra}'
            assert np.array_equal(c['rB'].astype(np.float32), rb.astype(np.float32))
    assert len(contacts) == total and total > 300


def _random_boxes(n=3000, seed=11):
    rand = lcg(seed)
    s = Scene('boxes')
    s.params.iterations = 0
    for i in range(n):
        big = i % 499 == 0
        size = [30, 30, 1] if big else [0.3 + rand(), 0.3 + rand(), 0.3 + rand()]
        k = s.box(size, 1 if rand() < 0.9 else 0, 0.5, [(rand() - 0.5) * 40, (rand() - 0.5) * 40, (rand() - 0.5) * 40])
        if not big:
            s.bodies[k].rot = qnormalize([rand() - 0.5, rand() - 0.5, rand() - 0.5, rand() - 0.5])
    s.ignore(2, 1)
    return s


def test_broadphase_pair_set_bit_exact(cuda_lib):
    """avbd3d-gpu.gpu.test.ts:144-205: 3000 random boxes with large ones and an ignored pair; the
    GPU's pairs are exactly the oracle's rule set (f32 tests, bit for bit)."""
    s = _random_boxes()
    w = avbd_b200.CudaSolver3D(s)
    w.step()
    got = {tuple(p) for p in w.read_pairs().tolist()}
    assert w.read_counters()['overflow'] == 0
    want = {tuple(p) for p in Oracle(s).pairs().tolist()}
    assert got == want, f'{len(got ^ want)} pairs differ'
    assert (2, 1) not in got and len(got) > 100


def _graph_from(manifolds, n, dynamic, joints_info=()):
    nbr = [[] for _ in range(n)]
    for m in manifolds:
        a, b = int(m['a']), int(m['b'])
        if dynamic[a] and dynamic[b]:
            nbr[a].append(b)
            nbr[b].append(a)
    for t, a, b in joints_info:
        if a >= 0 and dynamic[a] and dynamic[b]:
            nbr[a].append(b)
            nbr[b].append(a)
    start = np.zeros(n + 1, dtype=np.int32)
    for i in range(n):
        start[i + 1] = start[i] + len(nbr[i])
    flat = np.array([j for i in range(n) for j in nbr[i]], dtype=np.int32)
    return start, flat


def test_colouring_bit_exact(cuda_lib):
    """Jones-Plassmann colouring (wgsl-topology.ts:155-328): the GPU's colour state after each step is
    the oracle's colouring of the GPU's own constraint graph from the previous state, bit for bit."""
    s = drop_pile(4000, seed=2, spacing=1.6, layers=6)
    w = avbd_b200.CudaSolver3D(s)
    n = len(s.bodies)
    dynamic = np.array([b.mass > 0 for b in s.bodies], dtype=np.uint8)
    state = np.full(n, NO_COLOR, dtype=np.uint32)
    checked = 0
    for step in range(40):
        w.step()
        man, _ = w.read_contacts()
        got = w.read_colors()
        start, flat = _graph_from(man, n, dynamic)
        want, stats = color_graph(n, dynamic, start, flat, state, 64, 32)
        assert np.array_equal(got[dynamic == 1], want[dynamic == 1]), f'step {step}: {(got != want).sum()} colours differ'
        c = w.read_counters()
        assert c['colors'] == stats['colors'] and c['clashes'] == stats['clashes'] and c['rounds'] == stats['rounds'], (c, stats)
        state = got
        checked += len(man)
    assert checked > 1000


def test_pyramid_coloured_step_matches_fp64(cuda_lib):
    """Config 1, the 210-cube pyramid (more than 64 bodies: coloured mode): from the oracle's state
    rounded to f32, with the oracle's colouring, one GPU step against one FP64 step of the GPU-mode
    oracle. Poses within 1e-5; every multiplier row (normal and both friction rows) within 1e-5
    relative plus the stated floor."""
    scene = cube_pyramid(20)
    o = Oracle(scene)
    for _ in range(90):
        o.step_gpu()
    o.round_f32()
    w = cuda_from_oracle(o, scene.params)
    o.step_gpu()
    w.set_fixed_colors(o.colors())
    w.step()
    d = pose_diff(w.read_bodies(), o.bodies())
    gm, om = contact_map(*w.read_contacts()), oracle_contact_map(o)
    lp = lambda_parity(gm, om)
    print(f'pyramid coloured step: pose diff {d:.3e}, {len(gm)} contacts, lambda {lp}')
    assert d < 1e-5
    assert set(gm) == set(om) and lp['ratio'] <= 1.0


def test_determinism_bitwise(cuda_lib):
    """avbd3d-gpu.gpu.test.ts:442-491: a pile run twice ends in the same bits."""
    s = drop_pile(20000, seed=4, spacing=1.6, layers=8)
    runs = []
    for _ in range(2):
        w = avbd_b200.CudaSolver3D(s)
        w.step(90)
        runs.append(w.read_bodies().view(np.uint32).copy())
        c = w.read_counters()
        assert c['overflow'] == 0 and c['error'] == 0 and c['manifolds'] > 1000
        w.destroy()
    assert np.array_equal(runs[0], runs[1])


def test_graph_replay_matches_direct_launches(cuda_lib):
    """A step replayed from a captured CUDA graph does exactly what the direct launches do."""
    s = drop_pile(6000, seed=6, spacing=1.6, layers=6)
    out = []
    for graphs in (True, False):
        w = avbd_b200.CudaSolver3D(s)
        w.use_graphs(graphs)
        w.enable_step_stats(64)
        w.step(70)
        c = w.read_counters()
        assert c['graphs'] == (1 if graphs else 0) and c['error'] == 0
        st = w.read_step_stats()
        assert len(st) == 64 and np.all(st['solve_ms'] > 0) and st['manifolds'][-1] > 500
        out.append(w.read_bodies().view(np.uint32).copy())
        w.destroy()
    assert np.array_equal(out[0], out[1])


def test_pivot_floor_keeps_sliver_finite(cuda_lib):
    """tests-gpu/pivot.gpu.test.ts:15-40: a light sliver on its edge under PENALTY_MAX contacts stays finite."""
    s = Scene('sliver')
    s.box([100, 100, 1], 0, 0.8, [0, 0, -0.5])
    chip = s.box([0.05, 0.004, 0.004], 750, 0.8, [0, 0, 0.004 * math.sqrt(0.5)])
    sn = math.sin(math.pi / 8)
    s.bodies[chip].rot = [sn, 0.0, 0.0, math.cos(math.pi / 8)]
    o = Oracle(s)
    o.step(5)
    man, _ = o.manifolds()
    assert any(int(m[3]) == 2 for m in man)
    o.set_contact_penalty(1e10)
    rec = o.body(chip)
    rec[10:13] = [3, 0, 0]
    o.set_body(chip, rec)
    w = cuda_from_oracle(o, s.params)
    w.step(20)
    b = w.read_bodies()[chip]
    state = np.concatenate([b[f].ravel() for f in b.dtype.names]).astype(np.float64)
    assert np.all(np.isfinite(state))
    assert abs(b['pos'][2]) < 0.05 and math.hypot(b['pos'][0], b['pos'][1]) < 0.05


JOINT_CASES = [
    dict(name='rigid', yield_force=math.inf, fracture=math.inf),
    dict(name='yields', yield_force=30, fracture=math.inf),
    dict(name='fracture below the force asked', yield_force=30, fracture=40),
    dict(name='yield above the force asked', yield_force=200, fracture=math.inf),
    dict(name='yields between yield and fracture', yield_force=30, fracture=200),
    dict(name='within bend limit', yield_force=30, fracture=200, break_bend=0.065),
    dict(name='past bend limit', yield_force=30, fracture=200, break_bend=0.05),
    dict(name='rest', yield_force=math.inf, fracture=math.inf, rest=[math.sin(25 * math.pi / 360), 0, 0, math.cos(25 * math.pi / 360)]),
]


@pytest.mark.parametrize('case', JOINT_CASES, ids=[c['name'] for c in JOINT_CASES])
def test_joint_yield_fracture_rest(cuda_lib, case):
    """avbd3d-gpu.gpu.test.ts:992-1058: plastic, breaking and rest joints decide as the reference does."""
    s = Scene('joint')
    s.params.gravity = 0.0
    a = s.box([1, 1, 1], 0, 0.5, [0, 0, 5])
    b = s.box([1, 1, 1], 10, 0.5, [1, 0, 5])
    if case.get('rest'):
        s.bodies[b].rot = list(case['rest'])
        s.bodies[b].pos = [0.5 + 0.5 * math.cos(25 * math.pi / 180), -0.5 * math.sin(25 * math.pi / 180), 5]
    s.bodies[b].ang_vel = [0, 10, 0]
    j = s.joint(a, b, [0.5, 0, 0], [-0.5, 0, 0], math.inf, math.inf, case['fracture'])
    f = s.forces[j]
    f.yield_force = case['yield_force']
    f.break_bend = case.get('break_bend', math.inf)
    if case.get('rest'):
        f.rest = list(case['rest'])
    f.penalty_ang = [100.0] * 3
    f.penalty_lin = [1e4] * 3
    o = Oracle(s)
    w = cuda_from_oracle(o, s.params)
    w.set_fixed_colors(oracle_sequential_colors(o))
    w.step()
    o.step()
    recs, _ = w.read_joints()
    ref = o.force(0) if o.force_count else None
    assert ref is not None
    broken_ref = ref[26] != 0
    broken_gpu = recs[0]['stiffness_lin'] == 0 and recs[0]['stiffness_ang'] == 0
    assert broken_gpu == broken_ref, case['name']
    if not broken_ref:
        assert abs(np.linalg.norm(recs[0]['lam_ang']) - np.linalg.norm(ref[12:15])) < 0.02 * max(1, np.linalg.norm(ref[12:15]))
        for r in range(3):
            assert abs(recs[0]['pen_ang'][r] - ref[6 + r]) < 1e-3 * max(1, recs[0]['pen_ang'][r])
    d = pose_diff(w.read_bodies(), o.bodies())
    assert d < 1e-5, f'{case["name"]}: pose diff {d}'
