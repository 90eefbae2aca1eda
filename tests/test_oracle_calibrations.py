"""The reference CPU solver's own behaviour tests (tests/avbd3d-ref.test.ts:62-170), run on the
oracle: Coulomb stopping distances, static friction on the ramp, the spring's equilibrium, hard
joints holding, fracture, a world-anchored drag joint, finite states at 1 and 20 iterations,
determinism and box mass properties. No GPU."""

import math

import numpy as np

from avbd_b200.scenes import DEMO_SCENES, Scene, demo_scene
from oracle import K_JOINT, Oracle


def _run(name: str, frames: int, iterations: int | None = None) -> Oracle:
    s = demo_scene(name)
    if iterations is not None:
        s.params.iterations = iterations
    o = Oracle(s)
    o.step(frames)
    return o


def _rotate(q, v):
    u, w = np.asarray(q[:3]), q[3]
    v = np.asarray(v, dtype=np.float64)
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def _joint_error(o: Oracle, i: int) -> float:
    """|pA - pB| of joint i (forces.ts:150-155; rA is a world point when there is no body A)."""
    r = o.force(i)
    b = o.bodies()
    a, bb = int(r[1]), int(r[2])
    pa = r[39:42] if a < 0 else b[a, 0:3] + _rotate(b[a, 3:7], r[39:42])
    pb = b[bb, 0:3] + _rotate(b[bb, 3:7], r[42:45])
    return float(np.linalg.norm(pa - pb))


def _joints(o: Oracle):
    return [i for i in range(o.force_count) if int(o.force(i)[0]) == K_JOINT]


def test_dynamic_friction_stopping_distance():
    """:62-75: boxes launched at 10 m/s along x stop where Coulomb friction says (15 %)."""
    b = _run('Dynamic Friction', 300).bodies()
    for i in range(11):
        slid = b[1 + i, 0]
        if i == 10:
            assert abs(slid - 50) < 1e-6  # the frictionless box keeps its speed
            continue
        mu = math.sqrt((5 - i * 0.5) * 0.5)
        expected = 100 / (2 * mu * 10)
        assert abs(slid - expected) / expected < 0.15, (i, slid, expected)


def test_static_friction_on_the_ramp():
    """:77-91: boxes above tan(30°) hold on the ramp, the rest slide off."""
    o = _run('Static Friction', 600)
    xs = o.bodies()[2:, 0].copy()
    o.step(120)
    b = o.bodies()[2:]
    for i in range(len(b)):
        mu = math.sqrt((i / 10) * 0.25 + 0.25)
        if mu > math.tan(math.pi / 6) + 0.01:
            assert b[i, 2] > 7 and abs(b[i, 0] - xs[i]) < 0.005, (i, mu)
        elif mu < math.tan(math.pi / 6) - 0.01:
            assert b[i, 2] < 1.5, (i, mu)


def test_spring_equilibrium():
    """:93-102: anchor at z 14, rest length 4, k 100, mass 8: the block oscillates about z 9.2."""
    o = _run('Spring', 600)
    total = 0.0
    for _ in range(600):
        o.step()
        total += o.bodies()[2, 2]
    assert abs(total / 600 - 9.2) < 0.05


def test_hard_joints_hold():
    """:104-118: once the swing has died down the ropes' and the bridge's joints hold."""
    for name, bound, frames in (('Rope', 0.02, 240), ('Heavy Rope', 0.03, 600), ('Bridge', 0.03, 240)):
        o = _run(name, frames)
        err = max(_joint_error(o, i) for i in _joints(o))
        assert err < bound, (name, err)


def test_breakable_joints_fracture():
    """:120-125: the breakable bridge starts with 10 joints and loses some, not all, by frame 120."""
    def live(o):
        return sum(1 for i in _joints(o) if o.force(i)[26] == 0)
    assert live(_run('Breakable', 1)) == 10
    n = live(_run('Breakable', 120))
    assert 0 < n < 10


def test_world_anchored_drag_joint():
    """:127-138: a joint from a world point to the box's point where a ray along +y from (0, -10, 1)
    enters it pulls the box to the target."""
    o = _run('Ground', 120)
    b = o.bodies()[1]
    x, q, half = b[0:3], b[3:7], b[16:19] / 2
    # the ray's entry into the box, in the box frame (slab test; Solver.pick)
    qi = np.array([-q[0], -q[1], -q[2], q[3]])
    origin, direction = _rotate(qi, np.array([0.0, -10.0, 1.0]) - x), _rotate(qi, [0.0, 1.0, 0.0])
    t0, t1 = -math.inf, math.inf
    for k in range(3):
        if abs(direction[k]) < 1e-12:
            assert abs(origin[k]) <= half[k]
            continue
        ta, tb = (-half[k] - origin[k]) / direction[k], (half[k] - origin[k]) / direction[k]
        t0, t1 = max(t0, min(ta, tb)), min(t1, max(ta, tb))
    assert t0 <= t1 and t0 > 0, 'the ray enters the box'
    local = origin + t0 * direction
    target = np.array([3.0, 2.0, 4.0])
    o.L.orc_add_joint(o.h, -1, 1, target.ctypes.data_as(_dp_type()), local.ctypes.data_as(_dp_type()), 5000.0, 0.0, math.inf)
    o.step(300)
    # (force indices move as manifolds come and go: find the joint by its bodies)
    k = [i for i in _joints(o) if int(o.force(i)[1]) == -1 and int(o.force(i)[2]) == 1]
    assert len(k) == 1
    assert _joint_error(o, k[0]) < 0.05


def _dp_type():
    import ctypes
    return ctypes.POINTER(ctypes.c_double)


def test_every_scene_finite_at_1_and_20_iterations():
    """:141-151: blow-ups show within a few dozen frames."""
    for iterations in (1, 20):
        for name, _ in DEMO_SCENES:
            b = _run(name, 40, iterations).bodies()
            assert np.isfinite(b[:, 0:7]).all(), (name, iterations)


def test_deterministic():
    """:153-157."""
    a, b = _run('Soft Body', 120).bodies(), _run('Soft Body', 120).bodies()
    assert np.array_equal(a[:, 0:7], b[:, 0:7])


def test_box_mass_properties():
    """:159-165: a 1 x 2 x 3 box of density 2."""
    s = Scene('mass')
    i = s.box([1, 2, 3], 2, 0.5, [0, 0, 0])
    b = s.bodies[i]
    assert b.mass == 12 and list(b.moment) == [13, 10, 5]
    assert abs(b.radius - math.hypot(0.5, 1, 1.5)) < 1e-15
