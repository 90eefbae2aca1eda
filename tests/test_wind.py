"""The wind on sails (wgsl-solve.ts:262-335, GpuParams3D windSpeed / windAngle / windGust /
windPressure): the GPU-mode oracle's restatement checked against the physics it models (CPU), and the
CUDA step against the oracle (GPU)."""

import math

import numpy as np
import pytest

from avbd_b200.scenes import Scene
from oracle import Oracle

FACE_DOWN = (0.0, 0.0, 0.0, 1.0)                                   # local z (the sail's normal) along world z
EDGE_ON = (math.sin(math.pi / 4), 0.0, 0.0, math.cos(math.pi / 4))  # local z along -y: the plate stands upright
FACING_Y = EDGE_ON


def _plate_scene(rotation, pressure=0.72, speed=0.0, angle=0.0, gust=0.0, gravity=-10.0, as_box=False):
    s = Scene('sail')
    s.params.gravity = gravity
    s.params.wind_speed, s.params.wind_angle, s.params.wind_gust, s.params.wind_pressure = speed, angle, gust, pressure
    if as_box:
        i = s.box([1.0, 1.0, 0.02], 25.0, 0.5, [0.0, 0.0, 50.0])
        s.bodies[i].rot = list(rotation)
    else:
        s.sail([1.0, 1.0, 0.02], 25.0, 0.5, [0.0, 0.0, 50.0], rotation)
    return s


def _run(scene, steps):
    o = Oracle(scene)
    for _ in range(steps):
        o.step_gpu()
    return o.bodies()


def test_still_air_holds_a_face_down_sail_near_its_terminal_speed():
    """Face down, 1 m x 1 m at 0.5 kg: k = 0.72 x 1 / 0.5 = 1.44 / m. The drag k v^2 / (1 + 2 dt k v)
    (implicit in the normal speed) balances g at v = dt g + sqrt((dt g)^2 + g / k) = 2.81 m/s (2.64 in
    the continuum limit). After 1 s the sail falls at that speed where a box of the same size falls at g t."""
    sail = _run(_plate_scene(FACE_DOWN), 60)[0]
    box = _run(_plate_scene(FACE_DOWN, as_box=True), 60)[0]
    dtg = 10.0 / 60.0
    terminal = dtg + math.sqrt(dtg * dtg + 10.0 / 1.44)
    assert abs(box[9] + 10.0) < 0.05          # free fall: v = g t
    assert abs(sail[9] + terminal) < 0.01 * terminal
    # edge on, only the skin friction (6 % of the coefficient) acts: much faster than face down, slower than free fall
    edge = _run(_plate_scene(EDGE_ON), 60)[0]
    assert -10.0 < edge[9] < -2.0 * terminal


def test_no_air_makes_a_sail_a_box():
    """wind_pressure 0 (the parity setting): a sail's trajectory is the box's, bit for bit."""
    a = _run(_plate_scene(EDGE_ON, pressure=0.0, speed=7.0, gust=0.4), 30)
    b = _run(_plate_scene(EDGE_ON, pressure=0.0, as_box=True), 30)
    assert np.array_equal(a[:, :13], b[:, :13])


def test_steady_wind_pushes_a_sail_downwind():
    """Weightless, no gusts, 5 m/s along +y on a sail facing y: it accelerates along +y towards the
    wind's speed and gains no sideways or vertical speed."""
    r = _run(_plate_scene(FACING_Y, speed=5.0, angle=math.pi / 2, gravity=0.0), 30)[0]
    vx, vy, vz = r[7:10]
    assert 0.5 < vy < 5.0
    assert abs(vx) < 1e-9 and abs(vz) < 1e-9


def _flags_in_wind(n=24, seed=3):
    """Sails of random sizes and orientations in a gusting wind, far apart (no contacts)."""
    rng = np.random.default_rng(seed)
    s = Scene('flags in wind')
    s.params.wind_speed, s.params.wind_angle, s.params.wind_gust, s.params.wind_pressure = 8.0, 0.6, 0.4, 0.72
    for k in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        size = [rng.uniform(0.5, 1.5), rng.uniform(0.5, 1.5), 0.02]
        pos = [3.0 * (k % 6), 3.0 * (k // 6), 40.0 + rng.uniform(0.0, 5.0)]
        s.sail(size, rng.uniform(10.0, 40.0), 0.5, pos, q, velocity=rng.normal(0.0, 1.0, 3))
    return s


@pytest.mark.gpu
def test_cuda_sails_in_gusting_wind_match_the_oracle(cuda_lib):
    """24 sails in an 8 m/s wind with gusts, 60 steps: the CUDA step (f32) against the GPU-mode oracle
    (FP64), poses within 1e-4 (60 steps of f32 rounding of positions near 40 m and of the gusts'
    phases), and every sail pushed along the wind."""
    import avbd_b200
    from _util import pose_diff
    scene = _flags_in_wind()
    w = avbd_b200.CudaSolver3D(scene)
    o = Oracle(scene)
    start = w.read_bodies().copy()
    for step in range(60):
        w.step()
        o.step_gpu()
    got = w.read_bodies()
    d = pose_diff(got, o.bodies())
    print(f'sails in wind, 60 steps: pose diff {d:.3e}')
    assert d < 1e-4
    wind = np.array([math.cos(0.6), math.sin(0.6), 0.0])
    assert np.all((got['pos'] - start['pos']) @ wind > 0.0)
    # the same sails without air: the wind is what moved them downwind
    calm = _flags_in_wind()
    calm.params.wind_pressure = 0.0
    c = avbd_b200.CudaSolver3D(calm)
    c.step(60)
    assert ((got['pos'] - c.read_bodies()['pos']) @ wind).mean() > 0.5
    w.destroy()
    c.destroy()


@pytest.mark.gpu
def test_batched_sails_in_wind_match_single_worlds(cuda_lib):
    """The wind in batched worlds: three worlds of sails in gusting wind step bit for bit as each alone
    with a one-block solve (the batch's scope), 30 steps; the world's step word sets the gusts' phase
    in each world."""
    import avbd_b200
    scenes = [_flags_in_wind(n=8, seed=s) for s in (4, 5, 6)]
    n = sum(len(s.bodies) for s in scenes)
    b = avbd_b200.BatchSolver3D(len(scenes), n, params=scenes[0].params)
    for s in scenes:
        b.add_scene(s)
    singles = [avbd_b200.CudaSolver3D(s) for s in scenes]
    for w in singles:
        w.set_solve_blocks(1)
    b.step(30)
    for w in singles:
        w.step(30)
    b.synchronize()
    for i, w in enumerate(singles):
        assert np.array_equal(b.read_bodies(i).view(np.uint32), w.read_bodies().view(np.uint32)), f'world {i}'
        w.destroy()
    b.destroy()
