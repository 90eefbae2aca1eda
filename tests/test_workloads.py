"""The synthetic workloads the bench runs hold the shapes, sizes and value distributions they are
specified with (the reference's own bench scenes are procedural too, bench-scenes.ts): the cube
pyramid (C1), the drop pile (C2), hulls and chains (C3), the batched worlds (C4) and the
differentiated worlds (C5). No GPU needed."""

import math

import numpy as np

from avbd_b200.scenes import SHAPE_SPHERE, batched_worlds, cube_pyramid, drop_pile, hulls_and_chains, tumbling_world


def _arrays(scene):
    mass = np.array([b.mass for b in scene.bodies])
    size = np.array([b.size for b in scene.bodies])
    shape = np.array([b.shape for b in scene.bodies])
    friction = np.array([b.friction for b in scene.bodies])
    return mass, size, shape, friction


def test_cube_pyramid_rows():
    s = cube_pyramid(20)
    mass, size, _, friction = _arrays(s)
    dyn = mass > 0
    assert dyn.sum() == 210 and (~dyn).sum() == 1
    assert np.all(size[dyn] == 1.0) and np.allclose(mass[dyn], 1.0) and np.all(friction[dyn] == 0.5)
    pos = np.array([b.pos for b in s.bodies])[dyn]
    for y in range(20):
        row = np.sort(pos[np.isclose(pos[:, 2], y + 0.5)][:, 0])
        assert len(row) == 20 - y
        assert np.allclose(row, np.arange(20 - y) * 1.01 + 0.5 * y - 10)


def test_drop_pile_distributions():
    n = 20000
    s = drop_pile(n, seed=1)
    mass, size, shape, friction = _arrays(s)
    dyn = mass > 0
    assert dyn.sum() == n and (~dyn).sum() == 1  # the static ground box
    sphere = (shape == SHAPE_SPHERE) & dyn
    box = (shape != SHAPE_SPHERE) & dyn
    assert abs(sphere.sum() / n - 0.3) < 0.015
    half = size[box] / 2
    assert half.min() >= 0.25 and half.max() <= 0.75 and abs(half.mean() - 0.5) < 0.01
    r = size[sphere][:, 0] / 2
    assert r.min() >= 0.2 and r.max() <= 0.6 and abs(r.mean() - 0.4) < 0.01
    density = np.concatenate([mass[box] / np.prod(size[box], axis=1), mass[sphere] / (4 / 3 * math.pi * r ** 3)])
    assert density.min() >= 0.5 - 1e-9 and density.max() <= 2.0 + 1e-9 and abs(density.mean() - 1.25) < 0.02
    f = friction[dyn]
    assert f.min() >= 0.3 and f.max() <= 0.8
    speed = np.linalg.norm(np.array([b.vel for b in s.bodies])[dyn], axis=1)
    assert speed.max() <= 1.0 and abs(speed.mean() - 0.5) < 0.01
    q = np.array([b.rot for b in s.bodies])[dyn]
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0)
    assert np.abs(q.mean(axis=0)).max() < 0.02  # no preferred orientation


def test_hulls_and_chains_structure():
    chains, hulls = 4, 60
    s = hulls_and_chains(hulls=hulls, chains=chains, links=50, seed=9, distinct=16)
    mass, size, shape, _ = _arrays(s)
    dyn = mass > 0
    hull = shape >= 3
    assert hull.sum() == hulls and np.all(dyn[hull])
    links = dyn & ~hull
    assert links.sum() == chains * 50 and np.allclose(size[links], [0.2, 0.2, 0.5])
    assert (~dyn).sum() == 1 + chains  # ground and one anchor per chain
    joints = [f for f in s.forces if f.kind == 'joint']
    assert len(joints) == chains * 50
    assert all(f.fracture == 1e4 and f.fracture_linear and f.stiffness_ang == 0.0 and math.isinf(f.stiffness_lin) for f in joints)
    assert len(set(shape[hull].tolist())) <= 16
    assert s.params.iterations == 15


def test_batched_world_sizes():
    worlds = batched_worlds(1024, seed=3)
    sizes = np.array([sum(1 for b in w.bodies if b.mass > 0) for w in worlds])
    assert sizes.min() >= 16 and sizes.max() <= 512
    assert abs(np.median(sizes) - 64) <= 3
    assert abs(np.std(np.log(sizes)) - 0.5) < 0.05
    assert all(sum(1 for b in w.bodies if b.mass == 0) == 1 for w in worlds)  # each on its own ground


def test_tumbling_world():
    s = tumbling_world(np.random.default_rng(500), 64)
    mass, size, shape, friction = _arrays(s)
    dyn = mass > 0
    assert dyn.sum() == 64 and np.allclose(size[dyn], 0.8) and np.all(shape[dyn] != SHAPE_SPHERE) and np.all(friction[dyn] == 0.5)
