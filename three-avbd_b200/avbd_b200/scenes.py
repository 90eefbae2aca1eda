"""Scene descriptions: the reference's body/joint construction rules and the synthetic workloads.

A `Scene` collects bodies and forces in creation order, exactly as the reference's CPU solver
does when a scene builder calls `new Rigid(...)`, `new Joint(...)` (src/avbd3d/ref/body.ts:32-54,
forces.ts:129-147, 331-342). Mass properties are computed in double with the reference's own
operation order, so the CPU oracle replays the reference's golden trajectories bit for bit and the
CUDA backend receives the same values rounded to f32 (as GpuSolver3D.pack does, gpu/solver.ts:1176-1212).

Z is up in every scene (the reference's demo scenes are z-up: src/avbd3d/ref/scenes.ts:1).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SHAPE_BOX = 0
SHAPE_SPHERE = 1
SHAPE_SAIL = 2
SHAPE_HULL = 3

INF = math.inf


# --- maths in the reference's operation order (src/avbd3d/ref/math.ts) -------------------------

def _rotate(q, v):
    ux, uy, uz, w = q
    tx = (uy * v[2] - uz * v[1]) * 2
    ty = (uz * v[0] - ux * v[2]) * 2
    tz = (ux * v[1] - uy * v[0]) * 2
    return [v[0] + tx * w + (uy * tz - uz * ty), v[1] + ty * w + (uz * tx - ux * tz), v[2] + tz * w + (ux * ty - uy * tx)]


def _normalize3(v):
    length = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return [v[0] / length, v[1] / length, v[2] / length]


def _rad(deg):
    return deg * 0.017453292519943295


@dataclass
class Body:
    """A rigid body as the reference's `Rigid` holds it (ref/body.ts:13-62), in double."""

    pos: list
    size: list
    mass: float
    moment: list
    friction: float
    radius: float
    rot: list = field(default_factory=lambda: [0.0, 0.0, 0.0, 1.0])
    vel: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    ang_vel: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    prev_vel: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    initial_pos: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    initial_rot: list = field(default_factory=lambda: [0.0, 0.0, 0.0, 1.0])
    inertial_pos: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    inertial_rot: list = field(default_factory=lambda: [0.0, 0.0, 0.0, 1.0])
    shape: int = SHAPE_BOX
    groups: int = 0xFFFFFFFF
    mask: int = 0xFFFFFFFF


@dataclass
class Force:
    """A joint, spring or ignore pair in creation order (ref/forces.ts)."""

    kind: str  # 'joint' | 'spring' | 'ignore'
    a: int  # -1: the world (joints only)
    b: int
    rA: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    rB: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    stiffness_lin: float = INF
    stiffness_ang: float = 0.0
    fracture: float = INF
    fracture_linear: bool = False
    yield_force: float = INF
    break_bend: float = INF
    rest: list | None = None
    rest_start: list | None = None
    spring_stiffness: float = 0.0
    spring_rest: float = -1.0
    penalty_lin: list = field(default_factory=lambda: [0.0, 0.0, 0.0])
    penalty_ang: list = field(default_factory=lambda: [0.0, 0.0, 0.0])


@dataclass
class Params:
    """SolverParams (ref/solver.ts:139-165) plus the GPU flags (gpu/solver.ts:174-231)."""

    dt: float = 1.0 / 60.0
    gravity: float = -10.0
    iterations: int = 10
    alpha: float = 0.99
    beta_lin: float = 10000.0
    beta_ang: float = 100.0
    gamma: float = 0.999
    contact_margin: float = 0.01
    match_nearest: bool = False
    face_bias: bool = False
    start_at_rest: bool = False
    mass_penalty: bool = False
    reuse_contacts: bool = False
    # the wind on sails (gpu/solver.ts:200-206): 0 pressure is still no air, as the CPU solver has none
    wind_speed: float = 0.0
    wind_angle: float = 0.0
    wind_gust: float = 0.4
    wind_pressure: float = 0.0


class Scene:
    def __init__(self, name: str = ""):
        self.name = name
        self.bodies: list[Body] = []
        self.forces: list[Force] = []
        self.params = Params()
        self.hull_words = np.zeros(0, dtype=np.uint32)  # hull buffer (gpu/solver.ts:313-338 layout)
        self.hull_offsets: list[int] = []  # header offset of each hull record, in upload order

    # Rigid constructor (ref/body.ts:32-54)
    def box(self, size, density, friction, position, velocity=(0.0, 0.0, 0.0)) -> int:
        sx, sy, sz = (float(s) for s in size)
        mass = sx * sy * sz * density
        moment = [((sy * sy + sz * sz) / 12) * mass, ((sx * sx + sz * sz) / 12) * mass, ((sx * sx + sy * sy) / 12) * mass]
        hx, hy, hz = sx * 0.5, sy * 0.5, sz * 0.5
        radius = math.sqrt(hx * hx + hy * hy + hz * hz)
        v = [float(x) for x in velocity]
        self.bodies.append(Body(pos=[float(p) for p in position], size=[sx, sy, sz], mass=mass, moment=moment, friction=float(friction),
                                radius=radius, vel=list(v), prev_vel=list(v)))
        return len(self.bodies) - 1

    # A sail (src/avbd3d/shapes.ts:17-25): a thin box whose local z faces catch the wind (the GPU solver's
    # wind; the CPU solver has no air and treats it as a box)
    def sail(self, size, density, friction, position, rotation=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0)) -> int:
        i = self.box(size, density, friction, position, velocity)
        self.bodies[i].rot = [float(x) for x in rotation]
        self.bodies[i].shape = SHAPE_SAIL
        return i

    # A solid sphere (src/avbd3d/shapes.ts:83-91): a cubic box of side 2r with a sphere's mass properties
    def sphere(self, r, density, friction, position, velocity=(0.0, 0.0, 0.0)) -> int:
        i = self.box([2 * r, 2 * r, 2 * r], density, friction, position, velocity)
        b = self.bodies[i]
        b.mass = (4 / 3) * math.pi * r * r * r * density if density > 0 else 0.0
        inertia = 0.4 * b.mass * r * r
        b.moment = [inertia, inertia, inertia]
        b.radius = float(r)
        b.shape = SHAPE_SPHERE
        return i

    def add_hull_shape(self, shape) -> int:
        """Appends a hull record (a hulls.HullShape) to the scene's hull buffer; its header offset."""
        from .hulls import relocate
        at = len(self.hull_words) // 4
        self.hull_words = np.concatenate([self.hull_words, relocate(shape.packed, at)])
        self.hull_offsets.append(at)
        return at

    # A convex hull body (src/avbd3d/shapes.ts:58-70): principal frame at `position`, turned by `rotation`
    def hull(self, shape, density, friction, position, rotation=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0), offset=None) -> int:
        at = self.add_hull_shape(shape) if offset is None else int(offset)
        i = self.box(list(shape.size), density, friction, position, velocity)
        b = self.bodies[i]
        b.rot = [float(x) for x in rotation]
        b.mass = shape.volume * density if density > 0 else 0.0
        b.moment = [m * max(density, 0.0) for m in shape.moments]
        b.radius = float(shape.radius)
        b.shape = SHAPE_HULL + at
        return i

    def joint(self, a, b, rA, rB, stiffness_lin=INF, stiffness_ang=0.0, fracture=INF) -> int:
        self.forces.append(Force('joint', a, b, [float(x) for x in rA], [float(x) for x in rB], stiffness_lin, stiffness_ang, fracture))
        return len(self.forces) - 1

    def spring(self, a, b, rA, rB, stiffness, rest=-1.0) -> int:
        f = Force('spring', a, b, [float(x) for x in rA], [float(x) for x in rB])
        f.spring_stiffness = float(stiffness)
        f.spring_rest = float(rest)
        if f.spring_rest < 0:  # forces.ts:337-341
            A, B = self.bodies[a], self.bodies[b]
            pa = [x + y for x, y in zip(_rotate(A.rot, f.rA), A.pos)]
            pb = [x + y for x, y in zip(_rotate(B.rot, f.rB), B.pos)]
            d = [pa[k] - pb[k] for k in range(3)]
            f.spring_rest = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        self.forces.append(f)
        return len(self.forces) - 1

    def ignore(self, a, b) -> int:
        self.forces.append(Force('ignore', a, b))
        return len(self.forces) - 1

    @property
    def dynamic_count(self) -> int:
        return sum(1 for b in self.bodies if b.mass > 0)


# --- The demo scenes (src/avbd3d/ref/scenes.ts:8-258), in their order -------------------------

def _ground(s: Scene, z=0.0):
    return s.box([100, 100, 1], 0, 0.5, [0, 0, z])


def scene_empty(s):
    pass


def scene_ground(s):
    _ground(s)
    s.box([1, 1, 1], 1, 0.5, [0, 0, 4])


def scene_dynamic_friction(s):
    _ground(s)
    for x in range(11):
        s.box([1, 1, 0.5], 1, 5 - (x / 10) * 5, [0, -30 + x * 2, 0.75], [10, 0, 0])


def scene_static_friction(s):
    _ground(s)
    angle = _rad(30)
    ramp = s.box([40, 24, 1], 0, 1, [0, 0, 3])
    rot = [0.0, math.sin(angle * 0.5), 0.0, math.cos(angle * 0.5)]
    s.bodies[ramp].rot = rot
    tangent = _normalize3(_rotate(rot, [1, 0, 0]))
    normal = _normalize3(_rotate(rot, [0, 0, 1]))
    for i in range(11):
        friction = (i / 10) * 0.25 + 0.25
        y = -10 + i * 2
        rp = s.bodies[ramp].pos
        pos = [rp[k] + tangent[k] * -12 for k in range(3)]
        pos[1] += y
        pos = [pos[k] + normal[k] * 1.05 for k in range(3)]
        s.box([1, 1, 1], 1, friction, pos)


def scene_pyramid(s, size=16):
    _ground(s, -0.5)
    for y in range(size):
        for x in range(size - y):
            s.box([1, 0.5, 0.5], 1, 0.5, [x * 1.01 + y * 0.5 - size / 2, 0, y * 0.85 + 0.5])


def scene_rope(s):
    _ground(s, -20)
    prev = None
    for i in range(20):
        curr = s.box([1, 0.5, 0.5], 0 if i == 0 else 1, 0.5, [i, 0, 10])
        if prev is not None:
            s.joint(prev, curr, [0.5, 0, 0], [-0.5, 0, 0])
        prev = curr


def scene_heavy_rope(s):
    N, SIZE = 20, 5
    _ground(s, -20)
    prev = None
    for i in range(N):
        last = i == N - 1
        curr = s.box([SIZE, SIZE, SIZE] if last else [1, 0.5, 0.5], 0 if i == 0 else 1, 0.5, [i + (SIZE / 2 if last else 0), 0, 10])
        if prev is not None:
            s.joint(prev, curr, [0.5, 0, 0], [-SIZE / 2, 0, 0] if last else [-0.5, 0, 0])
        prev = curr


def scene_spring(s):
    _ground(s)
    anchor = s.box([1, 1, 1], 0, 0.5, [0, 0, 14])
    block = s.box([2, 2, 2], 1, 0.5, [0, 0, 8])
    s.spring(anchor, block, [0, 0, 0], [0, 0, 0], 100, 4)


def scene_springs_ratio(s):
    N = 8
    _ground(s, -10)
    prev = None
    for i in range(N):
        x = (i - (N - 1) * 0.5) * 3
        curr = s.box([1, 0.75, 0.75], 0 if i in (0, N - 1) else 1, 0.5, [x, 0, 12])
        if prev is not None:
            s.spring(prev, curr, [0.5, 0, 0], [-0.5, 0, 0], 10 if i % 2 == 0 else 10000, 3)
        prev = curr


def scene_stack(s):
    _ground(s)
    for i in range(10):
        s.box([1, 1, 1], 1, 0.5, [0, 0, i * 1.5 + 1])


def scene_stack_ratio(s):
    thickness = 1
    s.box([100, 100, thickness], 0, 0.5, [0, 0, 0])
    top = thickness * 0.5
    size = 1
    for _ in range(4):
        half = size * 0.5
        cz = top + half
        s.box([size, size, size], 1, 0.5, [0, 0, cz])
        top = cz + half
        size *= 2


def scene_soft_body(s):
    _ground(s)
    Klin, Kang = 1000, 250
    W = D = H = 4
    N = 3
    size = 0.8
    half = size * 0.5
    baseZ, gap = 8, 2
    for i in range(N):
        stackZ = i * (H * size + gap)
        grid = [[[0] * H for _ in range(D)] for _ in range(W)]
        for x in range(W):
            for y in range(D):
                for z in range(H):
                    px = (x - (W - 1) * 0.5) * size
                    py = (y - (D - 1) * 0.5) * size
                    pz = baseZ + stackZ + z * size
                    grid[x][y][z] = s.box([size, size, size], 1, 0.5, [px, py, pz])
        for x in range(1, W):
            for y in range(D):
                for z in range(H):
                    s.joint(grid[x - 1][y][z], grid[x][y][z], [half, 0, 0], [-half, 0, 0], Klin, Kang)
        for x in range(W):
            for y in range(1, D):
                for z in range(H):
                    s.joint(grid[x][y - 1][z], grid[x][y][z], [0, half, 0], [0, -half, 0], Klin, Kang)
        for x in range(W):
            for y in range(D):
                for z in range(1, H):
                    s.joint(grid[x][y][z - 1], grid[x][y][z], [0, 0, half], [0, 0, -half], Klin, Kang)
        for x in range(1, W):
            for y in range(D):
                for z in range(1, H):
                    s.ignore(grid[x - 1][y][z - 1], grid[x][y][z])
                    s.ignore(grid[x][y][z - 1], grid[x - 1][y][z])
        for x in range(W):
            for y in range(1, D):
                for z in range(1, H):
                    s.ignore(grid[x][y - 1][z - 1], grid[x][y][z])
                    s.ignore(grid[x][y][z - 1], grid[x][y - 1][z])
        for x in range(1, W):
            for y in range(1, D):
                for z in range(H):
                    s.ignore(grid[x - 1][y - 1][z], grid[x][y][z])
                    s.ignore(grid[x][y - 1][z], grid[x - 1][y][z])


def scene_bridge(s):
    N = 40
    length, width, height = 1, 4, 0.5
    hl, hw = length * 0.5, width * 0.5
    _ground(s)
    prev = None
    for i in range(N):
        curr = s.box([length, width, height], 0 if i in (0, N - 1) else 1, 0.5, [i - N / 2, 0, 10])
        if prev is not None:
            s.joint(prev, curr, [hl, hw, 0], [-hl, hw, 0], INF, 0)
            s.joint(prev, curr, [hl, -hw, 0], [-hl, -hw, 0], INF, 0)
        prev = curr
    for x in range(N // 4):
        for y in range(N // 8):
            s.box([1, 1, 1], 1, 0.5, [x - N / 8, 0, y + 12])


def scene_breakable(s):
    N, M, brk = 10, 5, 90
    _ground(s)
    prev = None
    for i in range(N + 1):
        curr = s.box([1, 1, 0.5], 1, 0.5, [i - N / 2, 0, 6])
        if prev is not None:
            s.joint(prev, curr, [0.5, 0, 0], [-0.5, 0, 0], INF, INF, brk)
        prev = curr
    s.box([1, 1, 5], 0, 0.5, [-N / 2, 0, 2.5])
    s.box([1, 1, 5], 0, 0.5, [N / 2, 0, 2.5])
    for i in range(M):
        s.box([2, 1, 1], 1, 0.5, [0, 0, i * 2 + 8])


DEMO_SCENES = [
    ('Empty', scene_empty), ('Ground', scene_ground), ('Dynamic Friction', scene_dynamic_friction),
    ('Static Friction', scene_static_friction), ('Pyramid', scene_pyramid), ('Rope', scene_rope),
    ('Heavy Rope', scene_heavy_rope), ('Spring', scene_spring), ('Spring Ratio', scene_springs_ratio),
    ('Stack', scene_stack), ('Stack Ratio', scene_stack_ratio), ('Soft Body', scene_soft_body),
    ('Bridge', scene_bridge), ('Breakable', scene_breakable),
]


def demo_scene(name: str) -> Scene:
    for n, build in DEMO_SCENES:
        if n == name:
            s = Scene(n)
            build(s)
            return s
    raise KeyError(name)


# --- Synthetic workloads -------------------------------------------------------------------------

def cube_pyramid(layers: int = 20, gravity: float = -9.81) -> Scene:
    """Unit-cube pyramid: `layers` rows (210 cubes at 20), density 1, friction 0.5, on a static
    ground box; row y holds layers - y cubes at x = i*1.01 + 0.5*y - layers/2, one row per metre."""
    s = Scene(f'cube pyramid {layers}')
    s.params.gravity = gravity
    _ground(s, -0.5)
    for y in range(layers):
        for x in range(layers - y):
            s.box([1, 1, 1], 1, 0.5, [x * 1.01 + y * 0.5 - layers / 2, 0, y * 1.0 + 0.5])
    return s


def _unit_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.standard_normal((n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def drop_pile(n: int = 100_000, seed: int = 1, spacing: float = 2.7, gravity: float = -9.81, layers: int = 10) -> Scene:
    """The large drop pile: `n` bodies on a jittered lattice `layers` deep, uniform random
    orientations, speed U[0, 1] m/s in a random direction; 70 % boxes (half-extents U[0.25, 0.75]),
    30 % spheres (radius U[0.2, 0.6]), density U[0.5, 2], friction U[0.3, 0.8]; a static ground box
    under them. Seeded (numpy PCG64)."""
    rng = np.random.default_rng(seed)
    s = Scene(f'drop pile {n}')
    s.params.gravity = gravity
    per_layer = math.ceil(n / layers)
    side = math.ceil(math.sqrt(per_layer))
    extent = side * spacing
    s.box([extent + 20.0, extent + 20.0, 1.0], 0, 0.5, [0.0, 0.0, -0.5])
    idx = np.arange(n)
    gx = idx % side
    gy = (idx // side) % side
    gz = idx // (side * side)
    jitter = rng.uniform(-0.05, 0.05, (n, 3))
    pos = np.stack([(gx - (side - 1) / 2) * spacing, (gy - (side - 1) / 2) * spacing, 1.5 + gz * spacing], axis=1) + jitter
    quats = _unit_quaternions(rng, n)
    dirs = rng.standard_normal((n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    vel = dirs * rng.uniform(0, 1, (n, 1))
    is_sphere = rng.uniform(0, 1, n) < 0.3
    half = rng.uniform(0.25, 0.75, (n, 3))
    radius = rng.uniform(0.2, 0.6, n)
    density = rng.uniform(0.5, 2.0, n)
    friction = rng.uniform(0.3, 0.8, n)
    for i in range(n):
        if is_sphere[i]:
            b = s.sphere(float(radius[i]), float(density[i]), float(friction[i]), pos[i].tolist(), vel[i].tolist())
        else:
            b = s.box((2 * half[i]).tolist(), float(density[i]), float(friction[i]), pos[i].tolist(), vel[i].tolist())
            s.bodies[b].rot = quats[i].tolist()
        if is_sphere[i]:
            s.bodies[b].rot = quats[i].tolist()
    return s


def small_world(rng: np.random.Generator, n: int, gravity: float = -9.81) -> Scene:
    """One world of the batched workload: a stack (columns of unit cubes) or a pile (jittered lattice
    of unit cubes and r = 0.5 spheres, random orientations), density 1, friction 0.5, on its own
    static ground box."""
    s = Scene(f'world {n}')
    s.params.gravity = gravity
    _ground(s, -0.5)
    if rng.uniform() < 0.5:
        cols = max(1, int(math.ceil(math.sqrt(n / 8))))
        placed = 0
        z = 0
        while placed < n:
            for c in range(cols * cols):
                if placed >= n:
                    break
                cx, cy = c % cols, c // cols
                s.box([1, 1, 1], 1, 0.5, [cx * 1.05 - cols / 2, cy * 1.05 - cols / 2, z * 1.0 + 0.5])
                placed += 1
            z += 1
    else:
        side = max(1, int(math.ceil((n / 3) ** 0.5)))
        q = _unit_quaternions(rng, n)
        for i in range(n):
            gx, gy, gz = i % side, (i // side) % side, i // (side * side)
            p = [(gx - side / 2) * 1.9 + rng.uniform(-0.05, 0.05), (gy - side / 2) * 1.9 + rng.uniform(-0.05, 0.05), 1.0 + gz * 1.9]
            if rng.uniform() < 0.3:
                b = s.sphere(0.5, 1, 0.5, p)
            else:
                b = s.box([1, 1, 1], 1, 0.5, p)
            s.bodies[b].rot = q[i].tolist()
    return s


def batched_worlds(count: int = 4096, seed: int = 3, median: int = 64, sigma: float = 0.5, lo: int = 16, hi: int = 512) -> list[Scene]:
    """The batched workload: `count` worlds whose dynamic body counts are round(lognormal(median,
    sigma)) clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.round(np.exp(np.log(median) + sigma * rng.standard_normal(count))), lo, hi).astype(int)
    return [small_world(rng, int(k)) for k in sizes]


def tumbling_world(rng: np.random.Generator, n: int = 64) -> Scene:
    """One world of the differentiated batch: `n` boxes tumbling and sliding on a plane."""
    s = Scene('tumbling')
    s.params.gravity = -9.81
    _ground(s, -0.5)
    side = int(math.ceil(math.sqrt(n)))
    q = _unit_quaternions(rng, n)
    for i in range(n):
        gx, gy = i % side, i // side
        p = [(gx - side / 2) * 1.6, (gy - side / 2) * 1.6, 0.6 + rng.uniform(0.0, 0.4)]
        v = [rng.uniform(-2, 2), rng.uniform(-2, 2), rng.uniform(0, 1)]
        b = s.box([0.8, 0.8, 0.8], 1, 0.5, p, v)
        s.bodies[b].rot = q[i].tolist()
        s.bodies[b].ang_vel = [rng.uniform(-3, 3) for _ in range(3)]
    return s


# --- convex hulls (config 3) ----------------------------------------------------------------------

def ellipsoid_hull(rng: np.random.Generator, points: int | None = None):
    """The hull of 8-32 points on an ellipsoid with semi-axes U[0.3, 1.0] (random orientation of the
    points' frame): the reference's convexHull of them (src/avbd3d/hull.ts)."""
    from .hulls import build_hull
    while True:
        k = int(points if points is not None else rng.integers(8, 33))
        axes = rng.uniform(0.3, 1.0, 3)
        d = rng.standard_normal((k, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        h = build_hull((d * axes).reshape(-1))
        if h is not None:
            return h


def hull_pairs(count: int = 200, seed: int = 5) -> Scene:
    """Overlapping pairs of a hull with a hull, a box or a sphere (either order), each pair far from
    the others; no gravity and no iterations, so one step's contacts are the narrowphase's."""
    rng = np.random.default_rng(seed)
    s = Scene('hull pairs')
    s.params.gravity = 0.0
    s.params.iterations = 0
    shapes = [ellipsoid_hull(rng) for _ in range(16)]
    offsets = [s.add_hull_shape(h) for h in shapes]
    for p in range(count):
        base = np.array([(p % 20) * 10.0, (p // 20) * 10.0, 0.0])
        kinds = [('hull', 'hull'), ('hull', 'box'), ('box', 'hull'), ('hull', 'sphere'), ('sphere', 'hull')][p % 5]
        for k, kind in enumerate(kinds):
            at = base if k == 0 else base + rng.uniform(-0.6, 0.6, 3)
            q = rng.standard_normal(4)
            q /= np.linalg.norm(q)
            if kind == 'hull':
                j = int(rng.integers(len(shapes)))
                i = s.hull(shapes[j], 1.0, 0.5, at.tolist(), q.tolist(), offset=offsets[j])
            elif kind == 'box':
                i = s.box(rng.uniform(0.4, 1.6, 3).tolist(), 1.0, 0.5, at.tolist())
                s.bodies[i].rot = q.tolist()
            else:
                i = s.sphere(float(rng.uniform(0.3, 0.8)), 1.0, 0.5, at.tolist())
    return s


def hull_pile(n: int = 300, seed: int = 7, spacing: float = 1.9, boxes: float = 0.2, spheres: float = 0.1, gravity: float = -9.81) -> Scene:
    """Hulls (ellipsoid point hulls), with some boxes and spheres, dropped on a jittered lattice onto a
    static ground box."""
    rng = np.random.default_rng(seed)
    s = Scene(f'hull pile {n}')
    s.params.gravity = gravity
    side = max(1, int(math.ceil(math.sqrt(n / 4))))
    s.box([side * spacing + 20.0, side * spacing + 20.0, 1.0], 0, 0.5, [0.0, 0.0, -0.5])
    shapes = [ellipsoid_hull(rng) for _ in range(min(n, 64))]
    offsets = [s.add_hull_shape(h) for h in shapes]
    for i in range(n):
        gx, gy, gz = i % side, (i // side) % side, i // (side * side)
        p = [(gx - (side - 1) / 2) * spacing + rng.uniform(-0.05, 0.05), (gy - (side - 1) / 2) * spacing + rng.uniform(-0.05, 0.05),
             1.2 + gz * spacing]
        q = rng.standard_normal(4)
        q /= np.linalg.norm(q)
        u = rng.uniform()
        if u < boxes:
            k = s.box(rng.uniform(0.5, 1.2, 3).tolist(), 1.0, 0.5, p)
            s.bodies[k].rot = q.tolist()
        elif u < boxes + spheres:
            s.sphere(float(rng.uniform(0.3, 0.6)), 1.0, 0.5, p)
        else:
            j = int(rng.integers(len(shapes)))
            s.hull(shapes[j], float(rng.uniform(0.5, 2.0)), float(rng.uniform(0.3, 0.8)), p, q.tolist(), offset=offsets[j])
    return s


def hulls_and_chains(hulls: int = 20000, chains: int = 1000, links: int = 50, seed: int = 9, distinct: int = 512) -> Scene:
    """Config 3: `hulls` hulls of 8-32 points on ellipsoids (semi-axes U[0.3, 1.0]) falling onto
    `chains` chains of `links` boxes (0.2 x 0.2 x 0.5) joined by ball joints (break force 1e4 N on the
    linear force: breakOnPull), each hung from a static anchor; static ground box. 15 iterations.
    `distinct` hull shapes are built and shared."""
    rng = np.random.default_rng(seed)
    s = Scene(f'hulls {hulls} + chains {chains}x{links}')
    s.params.gravity = -9.81
    s.params.iterations = 15
    cside = int(math.ceil(math.sqrt(chains)))
    cspacing = 3.2
    extent = cside * cspacing
    top = links * 0.5 + 6.0
    s.box([extent + 20.0, extent + 20.0, 1.0], 0, 0.5, [0.0, 0.0, -0.5])
    for c in range(chains):
        x = (c % cside - (cside - 1) / 2) * cspacing
        y = (c // cside - (cside - 1) / 2) * cspacing
        anchor = s.box([0.4, 0.4, 0.2], 0, 0.5, [x, y, top + 0.1])
        prev, prev_off = anchor, [0.0, 0.0, -0.1]
        for k in range(links):
            z = top - 0.25 - 0.5 * k
            b = s.box([0.2, 0.2, 0.5], 1.0, 0.5, [x, y, z])
            j = s.joint(prev, b, prev_off, [0.0, 0.0, 0.25], stiffness_lin=INF, stiffness_ang=0.0, fracture=1e4)
            s.forces[j].fracture_linear = True
            prev, prev_off = b, [0.0, 0.0, -0.25]
    shapes = [ellipsoid_hull(rng) for _ in range(min(distinct, hulls))]
    offsets = [s.add_hull_shape(h) for h in shapes]
    hside = int(math.ceil(extent / 2.2))
    for i in range(hulls):
        gx, gy, gz = i % hside, (i // hside) % hside, i // (hside * hside)
        p = [(gx - (hside - 1) / 2) * 2.2 + rng.uniform(-0.1, 0.1), (gy - (hside - 1) / 2) * 2.2 + rng.uniform(-0.1, 0.1), top + 2.5 + gz * 2.2]
        q = rng.standard_normal(4)
        q /= np.linalg.norm(q)
        j = int(rng.integers(len(shapes)))
        s.hull(shapes[j], 1.0, float(rng.uniform(0.3, 0.8)), p, q.tolist(), offset=offsets[j])
    return s
