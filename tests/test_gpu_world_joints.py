"""World joints (appendWorldJoint / setWorldAnchor, gpu/solver.ts:1592-1623, 1937-1939) against the
FP64 oracle; joint slots released and reused (releaseJoints, appendConstraints, :1709-1771); and the
device storage views (bodyBuffer, contactStorage / contactStorages(), :638-650) read back through
torch and compared with the synchronous readbacks."""

import math

import numpy as np
import pytest

import avbd_b200
from avbd_b200 import _abi
from avbd_b200.scenes import Scene, demo_scene
from avbd_b200.solver import pack_force
from oracle import Oracle
from _util import cuda_from_oracle, joint_records, oracle_sequential_colors, pose_diff

pytestmark = pytest.mark.gpu

ANCHOR = [0.0, 0.0, 5.0]
LOCAL = [-0.5, 0.0, 0.0]


def _pendulum(world_joint: bool) -> Scene:
    """Two boxes on a ball joint, the first hung from the world point ANCHOR by its end LOCAL."""
    s = Scene('pendulum')
    a = s.box([1.0, 0.5, 0.5], 1.0, 0.5, [0.5, 0.0, 5.0])
    b = s.box([1.0, 0.5, 0.5], 1.0, 0.5, [1.5, 0.0, 5.0])
    s.bodies[a].vel = [0.0, 1.0, 0.0]
    s.joint(a, b, [0.5, 0.0, 0.0], [-0.5, 0.0, 0.0], math.inf, 0.0)
    if world_joint:
        s.joint(-1, a, ANCHOR, LOCAL, math.inf, 0.0)
    return s


def _anchor_error(bodies) -> float:
    """Distance of body 0's point LOCAL from ANCHOR."""
    q = bodies['rot'][0].astype(np.float64)
    v = np.array(LOCAL)
    u, s = q[:3], q[3]
    world = v + 2.0 * s * np.cross(u, v) + 2.0 * np.cross(u, np.cross(u, v)) + bodies['pos'][0]
    return float(np.linalg.norm(world - np.array(ANCHOR)))


def test_append_world_joint_matches_oracle(cuda_lib):
    o = Oracle(_pendulum(True))
    w = avbd_b200.CudaSolver3D(_pendulum(False))
    slot = w.append_world_joint(0, ANCHOR, LOCAL)
    assert slot == 1
    # the record is the one the reference packs for a Joint with no body A (forces.ts:129-147)
    recs, info = w.read_joints()
    ref, ref_info, _ = joint_records(o)
    assert (int(info[1]['type']), int(info[1]['a']), int(info[1]['b'])) == (int(ref_info[1]['type']), -1, 0)
    for f in ('stiffness_lin', 'stiffness_ang', 'fracture', 'torque_arm', 'yield_force', 'break_bend', 'rest', 'rest_start', 'r_a', 'r_b',
              'pen_lin', 'pen_ang', 'lam_lin', 'lam_ang'):
        assert np.array_equal(np.asarray(recs[1][f], np.float32), np.asarray(ref[1][f], np.float32)), f
    w.set_fixed_colors(oracle_sequential_colors(o))
    w.step()
    o.step()
    d1 = pose_diff(w.read_bodies(), o.bodies())
    for _ in range(59):
        w.step()
        o.step()
    b = w.read_bodies()
    d60 = pose_diff(b, o.bodies())
    err = _anchor_error(b)
    print(f'world joint: pose diff after 1 step {d1:.2e}, after 60 steps {d60:.2e} (FP32 against FP64); anchor error {err:.2e} m')
    assert d1 < 1e-5  # one step from the same state, as the seeded single-step tests
    assert d60 < 1e-2 and err < 0.05
    c = w.read_counters()
    assert c['error'] == 0
    w.destroy()


def test_set_world_anchor_matches_oracle(cuda_lib):
    scene = _pendulum(True)
    o = Oracle(scene)
    o.step(20)
    w = cuda_from_oracle(o, scene.params)
    moved = [0.3, 0.0, 5.2]
    w.set_world_anchor(1, moved)
    o.set_joint_anchor(1, moved)
    recs, _ = w.read_joints()
    assert np.array_equal(recs[1]['r_a'], np.float32(moved))
    w.set_fixed_colors(oracle_sequential_colors(o))
    w.step()
    o.step()
    d = pose_diff(w.read_bodies(), o.bodies())
    recs, _ = w.read_joints()
    c0 = o.force(1)[15:18]  # the step's C0 of the joint, from the moved world point
    print(f'moved anchor: pose diff {d:.2e}, C0 {recs[1]["c0_lin"][:3]} vs {c0}')
    assert d < 1e-5
    assert np.abs(recs[1]['c0_lin'][:3] - c0).max() < 1e-5
    assert np.abs(c0).max() > 0.05  # the step saw the moved point
    # invalid calls change nothing
    with pytest.raises(avbd_b200.AvbdError):
        w.set_world_anchor(7, moved)
    with pytest.raises(avbd_b200.AvbdError):
        w.set_world_anchor(1, [0.0, math.nan, 0.0])
    with pytest.raises(avbd_b200.AvbdError):
        w.append_world_joint(5, ANCHOR, LOCAL)
    with pytest.raises(avbd_b200.AvbdError):
        w.append_world_joint(0, [math.inf, 0.0, 0.0], LOCAL)
    recs2, _ = w.read_joints()
    assert len(recs2) == 2 and np.array_equal(recs2[1]['r_a'], np.float32(moved))
    w.destroy()


class _Device:
    """A device array by address, for torch.as_tensor."""

    def __init__(self, address: int, shape, typestr: str):
        self.__cuda_array_interface__ = {'shape': tuple(shape), 'typestr': typestr, 'data': (int(address), False), 'version': 2,
                                         'strides': None}


def _read(address, shape, typestr, np_dtype):
    import torch
    t = torch.as_tensor(_Device(address, shape, typestr), device='cuda:0')
    return t.cpu().numpy().view(np_dtype)


def test_storage_views_match_readbacks(cuda_lib):
    scene = demo_scene('Pyramid')
    w = avbd_b200.CudaSolver3D(scene)
    w.step(30)
    w.synchronize()
    bv = w.body_storage()
    assert bv['count'] == len(scene.bodies) and bv['capacity'] >= bv['count'] and all(bv['fields'])
    bodies = w.read_bodies()
    as_rows = bodies.view(np.float32).reshape(-1, 10, 4)
    for f in range(10):
        got = _read(bv['fields'][f], (bv['count'], 4), '<f4', np.float32)
        assert np.array_equal(got, as_rows[:, f, :]), f'body field {f}'

    def live(view):
        counters = _read(view['counters'], (view['count_word'] + 1,), '<i4', np.uint32)
        slots = int(counters[view['count_word']])
        assert 0 < slots <= view['pair_capacity']
        pairs = _read(view['pairs'], (slots, 4), '<i4', np.uint32)
        normals = _read(view['normals'], (slots, 4), '<f4', np.float32)
        points = _read(view['points'], (slots * 8, 16), '<i4', np.uint32)
        out = []
        for p in range(slots):
            count = int(pairs[p, 3] & 15)
            if count:
                out.append((int(pairs[p, 0]), int(pairs[p, 1]), normals[p].copy(), points[8 * p:8 * p + count].copy()))
        return out

    last = live(w.contact_storage(0))
    man, con = w.read_contacts()
    assert len(last) == len(man) and len(last) > 0
    for (a, b, normal, pts), m in zip(last, man):
        assert (a, b) == (int(m['a']), int(m['b']))
        assert np.array_equal(normal[:3], m['normal']) and normal[3] == m['friction']
        assert np.array_equal(pts, con[int(m['first']):int(m['first']) + int(m['count'])].view(np.uint32).reshape(-1, 16))
    # after one more step, the other storage holds what the last step wrote
    w.step()
    w.synchronize()
    before = live(w.contact_storage(1))
    assert len(before) == len(last)
    for x, y in zip(before, last):
        assert x[:2] == y[:2] and np.array_equal(x[2], y[2]) and np.array_equal(x[3], y[3])
    w.destroy()


def _row(joined):
    """Four overlapping boxes in a row, weightless; `joined` lists the (a, b) pairs held by joints."""
    s = Scene('row')
    s.params.gravity = 0.0
    for i in range(4):
        s.box([1.05, 1.0, 1.0], 1.0, 0.5, [float(i), 0.0, 5.0])
    for a, b in joined:
        s.joint(a, b, [0.5, 0.0, 0.0], [-0.5, 0.0, 0.0], math.inf, math.inf)
    return s


def test_released_slots_collide_again_and_are_reused(cuda_lib):
    w = avbd_b200.CudaSolver3D(_row([(0, 1), (1, 2), (2, 3)]))
    w.step()
    pairs = {tuple(sorted(p)) for p in w.read_pairs().tolist()}
    assert not pairs & {(0, 1), (1, 2), (2, 3)}  # joined neighbours do not collide
    w.release_joints([1, 1, 99])  # repeats and slots out of range are ignored
    w.release_joints([1])         # so is a slot already released
    recs, info = w.read_joints()
    assert (int(info[1]['type']), int(info[1]['a']), int(info[1]['b'])) == (_abi.T_NONE, -1, -1)
    assert not recs[1].tobytes().strip(b'\0')
    w.step()
    pairs = {tuple(sorted(p)) for p in w.read_pairs().tolist()}
    assert (1, 2) in pairs and not pairs & {(0, 1), (2, 3)}
    # the next append takes the freed slot, then new ones; its pair stops colliding
    s = _row([(0, 2), (1, 3)])
    recs_new = np.array([pack_force(f, s.bodies)[0] for f in s.forces])
    info_new = np.array([pack_force(f, s.bodies)[1] for f in s.forces])
    slots = w.append_joints(recs_new, info_new)
    assert slots.tolist() == [1, 3]
    w.step()
    pairs = {tuple(sorted(p)) for p in w.read_pairs().tolist()}
    assert (1, 2) in pairs
    assert w.read_counters()['error'] == 0
    w.destroy()


def test_reused_slot_steps_as_a_fresh_world(cuda_lib):
    """Releasing a slot and appending into it gives the world built with that joint in the slot."""
    a = avbd_b200.CudaSolver3D(_row([(0, 1), (1, 2), (2, 3)]))
    a.release_joints([1])
    s = _row([(1, 3)])
    slot = a.append_joints(np.array([pack_force(s.forces[0], s.bodies)[0]]), np.array([pack_force(s.forces[0], s.bodies)[1]]))
    assert slot.tolist() == [1]
    b = avbd_b200.CudaSolver3D(_row([(0, 1), (1, 3), (2, 3)]))
    ra, ia = a.read_joints()
    rb, ib = b.read_joints()
    assert ra.tobytes() == rb.tobytes() and ia.tobytes() == ib.tobytes()
    for w in (a, b):
        w.step(20)
    assert a.read_bodies().tobytes() == b.read_bodies().tobytes()
    assert a.read_joints()[0].tobytes() == b.read_joints()[0].tobytes()
    # disableConstraint keeps the slot taken
    a.disable_joints([1])
    recs, info = a.read_joints()
    assert int(info[1]['type']) == _abi.T_JOINT and recs[1]['stiffness_lin'] == 0.0
    assert a.append_joints(np.array([pack_force(s.forces[0], s.bodies)[0]]), np.array([pack_force(s.forces[0], s.bodies)[1]])).tolist() == [3]
    a.destroy()
    b.destroy()
