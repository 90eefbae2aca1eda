"""Per-body aux records (setBodyAux: gravity scale and damping rates, gpu/solver.ts:1814-1845,
wgsl-solve.ts:9-20, 297-305) and lifecycle bits (setLifecycle, gpu/solver.ts:2069-2076; a cold
body's joints start afresh, wgsl-solve.ts:247-253), through the C ABI, against the GPU-mode FP64
oracle with the same records: one step from the oracle's state, poses within 1e-5."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200.scenes import demo_scene, tumbling_world
from oracle import Oracle
from _util import cuda_from_oracle, pose_diff

pytestmark = pytest.mark.gpu


def test_aux_gravity_scale_and_damping_match_oracle(cuda_lib):
    scene = tumbling_world(np.random.default_rng(4), 12)
    o = Oracle(scene)
    for _ in range(40):
        o.step_gpu()
    w = cuda_from_oracle(o, scene.params)
    idx = [1, 2, 3, 4, 5, 6]
    scales = [0.0, 0.5, -1.0, 2.0, 1.0, 1.0]
    lin = [0.0, 0.0, 0.0, 0.5, 3.0, 0.0]
    ang = [0.0, 0.0, 0.0, 0.5, 0.0, 4.0]
    w.set_body_aux(idx, scales, lin, ang)
    for i, s, l, a in zip(idx, scales, lin, ang):
        o.set_body_aux(i, s, l, a)
    aux = w.read_body_aux()
    assert np.allclose(aux[idx], np.stack([scales, lin, ang, np.zeros(6)], axis=1))
    assert np.allclose(aux[0], [1, 0, 0, 0]) and np.allclose(aux[7:], [1, 0, 0, 0])
    o.step_gpu()
    w.set_fixed_colors(o.colors())
    w.step()
    d = pose_diff(w.read_bodies(), o.bodies())
    print(f'aux step: pose diff {d:.3e}')
    assert d < 1e-5
    # scales alone keep the rates
    w.set_body_aux([4], [0.25])
    assert np.allclose(w.read_body_aux()[4], [0.25, 0.5, 0.5, 0.0])


def test_weightless_and_damped_bodies(cuda_lib):
    """Gravity scale 0: a resting body in the air stays put; a linear rate r: speed decays by exp(-r dt)
    each step with no contact."""
    scene = tumbling_world(np.random.default_rng(5), 4)
    for b in scene.bodies[1:]:
        b.pos[2] += 20.0
        b.vel = [0.0, 0.0, 0.0]
        b.prev_vel = [0.0, 0.0, 0.0]
        b.ang_vel = [0.0, 0.0, 0.0]
    scene.bodies[2].vel = [3.0, 0.0, 0.0]
    scene.bodies[2].prev_vel = [3.0, 0.0, 0.0]
    w = avbd_b200.CudaSolver3D(scene)
    z0 = w.read_bodies()['pos'][1, 2]
    w.set_body_aux([1, 2], [0.0, 0.0], [0.0, 2.0], [0.0, 0.0])
    w.step(10)
    b = w.read_bodies()
    assert abs(b['pos'][1, 2] - z0) < 1e-6
    dt = scene.params.dt
    assert b['vel'][2, 0] == pytest.approx(3.0 * np.exp(-2.0 * dt * 10), rel=1e-4)
    w.destroy()


def test_cold_body_joints_start_afresh(cuda_lib):
    scene = demo_scene('Rope')
    o = Oracle(scene)
    for _ in range(30):
        o.step_gpu()
    w = cuda_from_oracle(o, scene.params)
    w.set_lifecycle(3, 4)
    o.set_lifecycle(3, 4)
    o.step_gpu()
    w.set_fixed_colors(o.colors())
    w.step()
    d = pose_diff(w.read_bodies(), o.bodies())
    print(f'cold step: pose diff {d:.3e}')
    assert d < 1e-5
    with pytest.raises(avbd_b200.AvbdError):
        w.set_lifecycle(3, 1)  # only the disabled and cold bits
    w.destroy()


def test_runs_without_rates_take_the_default_rates(cuda_lib):
    """setBodyAux without rates (gpu/solver.ts:1826-1845): a lone slot changes only its gravity
    scale; a run of consecutive slots gets whole records with the default rates (0)."""
    w = avbd_b200.CudaSolver3D(demo_scene('Stack'))
    w.set_body_aux([1, 2, 3, 5], [0.5] * 4, [1.0] * 4, [2.0] * 4)
    w.set_body_aux([1, 2, 5], [0.25, 0.75, 3.0])
    aux = w.read_body_aux()
    assert np.allclose(aux[1], [0.25, 0.0, 0.0, 0.0]) and np.allclose(aux[2], [0.75, 0.0, 0.0, 0.0])
    assert np.allclose(aux[3], [0.5, 1.0, 2.0, 0.0])
    assert np.allclose(aux[5], [3.0, 1.0, 2.0, 0.0])
    assert np.allclose(aux[4], [1.0, 0.0, 0.0, 0.0])  # untouched: the defaults
    w.destroy()


def test_filters_by_slot_list_equal_filters_by_range(cuda_lib):
    """setFilters(indices, groups, collidesWith) (gpu/solver.ts:1791-1801) over a list of slots in any
    order (runs and scattered slots) writes what a contiguous write of the same values writes."""
    scene = demo_scene('Pyramid')
    n = len(scene.bodies)
    rng = np.random.default_rng(4)
    groups = rng.integers(1, 4, n).astype(np.uint32)
    masks = np.where(rng.uniform(size=n) < 0.5, 0xFFFFFFFF, 0xFFFFFFFE).astype(np.uint32)
    a, b, c = (avbd_b200.CudaSolver3D(scene) for _ in range(3))
    a.set_filters(0, np.stack([groups, masks], axis=1))
    order = np.concatenate([np.arange(0, 10), 10 + rng.permutation(n - 10)])
    b.set_filters_at(order, groups[order], masks[order])
    # the bricks start 0.25 m above the ground: 60 steps bring the pyramid into contact
    for w in (a, b, c):
        w.step(60)
    pairs = [{tuple(p) for p in w.read_pairs().tolist()} for w in (a, b, c)]
    assert len(pairs[2]) > 0 and len(pairs[0]) > 0
    assert pairs[0] == pairs[1] and pairs[0] != pairs[2]
    assert a.read_bodies().tobytes() == b.read_bodies().tobytes()
    with pytest.raises(avbd_b200.AvbdError):
        b.set_filters_at([n], [1], [1])
    for w in (a, b, c):
        w.destroy()


def test_rewrite_bodies_by_slot_list_equals_range_writes(cuda_lib):
    """rewriteBodies(indices, bodies) (gpu/solver.ts:1774-1784): a list of slots in runs writes what
    range writes of the same records write; a bad record refuses the whole call."""
    scene = demo_scene('Pyramid')
    a, b = avbd_b200.CudaSolver3D(scene), avbd_b200.CudaSolver3D(scene)
    for w in (a, b):
        w.step(20)
    recs = a.read_bodies()
    idx = np.array([3, 4, 5, 6, 9, 20, 21])
    new = recs[idx].copy()
    new['pos'][:, 2] += 0.5
    new['vel'][:, 0] = 1.0
    a.write_bodies(3, new[:4])
    a.write_bodies(9, new[4:5])
    a.write_bodies(20, new[5:])
    b.write_bodies_at(idx, new)
    for w in (a, b):
        w.step(10)
    assert a.read_bodies().tobytes() == b.read_bodies().tobytes()
    bad = new.copy()
    bad['pos'][3, 0] = np.nan
    before = b.read_bodies().tobytes()
    with pytest.raises(avbd_b200.AvbdError):
        b.write_bodies_at(idx, bad)
    assert b.read_bodies().tobytes() == before
    for w in (a, b):
        w.destroy()
