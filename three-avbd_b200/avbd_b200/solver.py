"""`CudaSolver3D`: the host-side mirror of the reference's `GpuSolver3D` (src/avbd3d/gpu/solver.ts:598)
over the C ABI, with the members `World` calls (step, readBodies, readJoints, readCounters,
readContactList, readPairs, addBodies, appendJoints, setFilters, params, destroy) and the
validation surface the reference's parity tests use (seedFrom's imports, fixedColors,
sequentialColors).

Packing follows GpuSolver3D.pack / writeJoint (solver.ts:1176-1256): f64 scene values rounded to
f32, Infinity stored as BIG, a rewritten slot flagged so it starts without contact history.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from ._abi import (BODY_DTYPE, CONTACT_DTYPE, INFO_DTYPE, JOINT_DTYPE, MANIFOLD_DTYPE, NO_COLOR, AvbdError, Counters, Params, ptr, uptr)
from .scenes import SHAPE_SPHERE, Scene


def finite(x: float) -> float:
    """Infinity is never stored on the device: BIG stands for it (avbd2d/gpu/layout.ts:1-4, gpu/solver.ts:115)."""
    if x == math.inf:
        return float(_abi.BIG)
    if x == -math.inf:
        return -float(_abi.BIG)
    return float(x)


def pack_bodies(bodies, up=(0.0, 0.0, 1.0)) -> np.ndarray:
    """Scene bodies (f64) as device records (GpuSolver3D.pack, solver.ts:1176-1212)."""
    out = np.zeros(len(bodies), dtype=BODY_DTYPE)
    if not len(bodies):
        return out
    col = lambda name: np.array([getattr(b, name) for b in bodies], dtype=np.float64)
    out['pos'] = col('pos')
    out['friction'] = col('friction')
    out['rot'] = col('rot')
    out['initial_pos'] = col('initial_pos')
    out['flags'] = 1.0
    out['initial_rot'] = col('initial_rot')
    out['size'] = col('size')
    out['mass'] = col('mass')
    out['moment'] = col('moment')
    out['radius'] = col('radius')
    out['inertial_pos'] = col('inertial_pos')
    out['inertial_rot'] = col('inertial_rot')
    out['vel'] = col('vel')
    pv = col('prev_vel')
    out['prev_up_vel'] = pv[:, 0] * up[0] + pv[:, 1] * up[1] + pv[:, 2] * up[2]
    out['ang_vel'] = col('ang_vel')
    out['shape'] = col('shape')
    return out


def torque_arm(size_a, size_b) -> float:
    """forces.ts:145-146: |sA + sB|^2 (sA = 0 for the world)."""
    s = [size_a[k] + size_b[k] for k in range(3)]
    return s[0] * s[0] + s[1] * s[1] + s[2] * s[2]


def pack_force(f, bodies) -> tuple[np.ndarray, np.ndarray]:
    """A scene joint/spring as (record, info) (GpuSolver3D.writeJoint, solver.ts:1214-1247)."""
    rec = np.zeros(1, dtype=JOINT_DTYPE)[0]
    info = np.zeros(1, dtype=INFO_DTYPE)[0]
    if f.kind == 'joint':
        rec['pen_lin'] = f.penalty_lin
        rec['stiffness_lin'] = finite(f.stiffness_lin)
        rec['pen_ang'] = f.penalty_ang
        rec['stiffness_ang'] = finite(f.stiffness_ang)
        rec['fracture'] = -finite(f.fracture) if f.fracture_linear else finite(f.fracture)
        sa = bodies[f.a].size if f.a >= 0 else [0.0, 0.0, 0.0]
        rec['torque_arm'] = torque_arm(sa, bodies[f.b].size)
        rec['yield_force'] = finite(f.yield_force)
        rec['break_bend'] = finite(f.break_bend)
        rest = f.rest if f.rest is not None else [0.0, 0.0, 0.0, 1.0]
        rec['rest'] = rest
        rec['rest_start'] = f.rest_start if f.rest_start is not None else rest
        rec['r_a'] = f.rA
        rec['r_b'] = f.rB
        info['type'] = _abi.T_JOINT
    elif f.kind == 'spring':
        rec['stiffness_lin'] = f.spring_stiffness
        rec['r_a'] = f.rA
        rec['spring_rest'] = f.spring_rest
        rec['r_b'] = f.rB
        rec['rest'] = [0.0, 0.0, 0.0, 1.0]
        rec['rest_start'] = [0.0, 0.0, 0.0, 1.0]
        info['type'] = _abi.T_SPRING
    else:
        raise ValueError(f.kind)
    info['a'] = f.a
    info['b'] = f.b
    return rec, info


def morton_order(positions: np.ndarray) -> np.ndarray:
    """Body order along a Z curve of the starting positions, 10 bits per axis (solver.ts:462-485)."""
    lo = positions.min(axis=0)
    hi = positions.max(axis=0)
    q = np.minimum(1023, np.floor((positions - lo) / np.maximum(hi - lo, 1e-9) * 1024)).astype(np.uint64)

    def spread(x):
        x = x & 0x3FF
        x = (x | (x << 16)) & 0x30000FF
        x = (x | (x << 8)) & 0x300F00F
        x = (x | (x << 4)) & 0x30C30C3
        x = (x | (x << 2)) & 0x9249249
        return x

    code = spread(q[:, 0]) | (spread(q[:, 1]) << 1) | (spread(q[:, 2]) << 2)
    return np.lexsort((np.arange(len(code)), code))


def to_params(sp) -> Params:
    """A scenes.Params (the reference's SolverParams + GPU flags) as the C record; a Params passes through."""
    if isinstance(sp, Params):
        return sp
    flags = (_abi.FLAG_MATCH_NEAREST if sp.match_nearest else 0) | (_abi.FLAG_FACE_BIAS if sp.face_bias else 0) | \
            (_abi.FLAG_START_AT_REST if sp.start_at_rest else 0) | (_abi.FLAG_MASS_PENALTY if sp.mass_penalty else 0) | \
            (_abi.FLAG_REUSE_CONTACTS if getattr(sp, 'reuse_contacts', False) else 0)
    p = Params(dt=sp.dt, gravity=sp.gravity, alpha=sp.alpha, beta_lin=sp.beta_lin, beta_ang=sp.beta_ang, gamma=sp.gamma,
               contact_margin=sp.contact_margin, iterations=sp.iterations, flags=flags)
    p.up[0], p.up[1], p.up[2] = 0.0, 0.0, 1.0
    p.wind_speed, p.wind_angle = getattr(sp, 'wind_speed', 0.0), getattr(sp, 'wind_angle', 0.0)
    p.wind_gust, p.wind_pressure = getattr(sp, 'wind_gust', 0.4), getattr(sp, 'wind_pressure', 0.0)
    return p


def scene_records(scene: Scene, order=None):
    """A scene as C-ABI records: bodies (in `order`), joints and springs with their infos, and ignore
    pairs, with body indices mapped through `order` (GpuSolver3D's refToGpu)."""
    n = len(scene.bodies)
    order = np.arange(n) if order is None else np.asarray(order)
    gpu_index = np.empty(n, dtype=np.int64)
    gpu_index[order] = np.arange(n)
    bodies = pack_bodies([scene.bodies[i] for i in order])
    recs, infos, ignores = [], [], []
    for f in scene.forces:
        if f.kind == 'ignore':
            ignores.append((int(gpu_index[f.a]), int(gpu_index[f.b])))
            continue
        r, i = pack_force(f, scene.bodies)
        i['a'] = int(gpu_index[f.a]) if f.a >= 0 else -1
        i['b'] = int(gpu_index[f.b])
        recs.append(r)
        infos.append(i)
    return (bodies, np.array(recs, dtype=JOINT_DTYPE), np.array(infos, dtype=INFO_DTYPE),
            np.array(ignores, dtype=np.uint32).reshape(-1, 2))


class CudaSolver3D:
    """One world on one B200. Mirrors GpuSolver3D's construction from a scene (`new GpuSolver3D(device,
    ref, {spatialSort})`): bodies and joints are uploaded in creation order (or Morton order with
    `spatial_sort=True`; `gpu_index` maps scene indices, as refToGpu does)."""

    def __init__(self, scene: Scene | None = None, *, body_capacity: int | None = None, joint_capacity: int | None = None,
                 pair_capacity: int = 0, device: int = 0, spatial_sort: bool = False):
        self.lib = _abi.load()
        n = len(scene.bodies) if scene else 0
        nj = sum(1 for f in scene.forces if f.kind != 'ignore') if scene else 0
        cfg = _abi.Config(body_capacity=body_capacity or max(n, 1), joint_capacity=joint_capacity or max(nj, 16), pair_capacity=pair_capacity,
                          device=device)
        self.handle = ctypes.c_void_p()
        code = self.lib.avbd_world_create(ctypes.byref(cfg), ctypes.byref(self.handle))
        if code != _abi.AVBD_OK:
            raise _abi.error(code, 'avbd_world_create failed (a B200 with the CUDA library is required; there is no CPU fallback)')
        self.order = np.arange(n)
        self.gpu_index = np.arange(n)
        self.fixed_colors = None
        if scene is not None:
            self.params = scene.params
            if spatial_sort and n:
                self.order = morton_order(np.array([b.pos for b in scene.bodies]))
                self.gpu_index = np.empty(n, dtype=np.int64)
                self.gpu_index[self.order] = np.arange(n)
            self.add_scene_hulls(scene)
            bodies, joints, infos, ignores = scene_records(scene, self.order)
            self.add_bodies(bodies)
            if len(joints):
                self.add_joints(joints, infos)
            if len(ignores):
                self.add_ignore_pairs(ignores)

    # --- lifetime ---
    def destroy(self):
        if getattr(self, 'handle', None) and self.handle.value:
            self.lib.avbd_world_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _check(self, code: int):
        if code != _abi.AVBD_OK:
            msg = self.lib.avbd_last_error(self.handle)
            raise _abi.error(code, msg.decode() if msg else '')

    # --- params (GpuParams3D) ---
    @property
    def params(self):
        p = Params()
        self._check(self.lib.avbd_get_params(self.handle, ctypes.byref(p)))
        return p

    @params.setter
    def params(self, sp):
        """Accepts a scenes.Params (the reference's SolverParams + GPU flags) or a ctypes Params."""
        self._check(self.lib.avbd_set_params(self.handle, ctypes.byref(to_params(sp))))

    # --- scene edits ---
    def add_hull(self, packed: np.ndarray) -> int:
        """A hull record (header at vec4 0) into the world's hull buffer; its header offset (shape - 3)."""
        packed = np.ascontiguousarray(packed, dtype=np.uint32)
        at = ctypes.c_uint32()
        self._check(self.lib.avbd_add_hull(self.handle, uptr(packed), len(packed) // 4, ctypes.byref(at)))
        return at.value

    def release_hull(self, offset: int):
        """The record's run goes free for a later add_hull (refused while a body uses it)."""
        self._check(self.lib.avbd_release_hull(self.handle, offset))

    def hull_storage(self) -> dict:
        t, c, f = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self.lib.avbd_hull_storage(self.handle, ctypes.byref(t), ctypes.byref(c), ctypes.byref(f)))
        return {'top': t.value, 'capacity': c.value, 'largest_free': f.value}

    def add_scene_hulls(self, scene: Scene):
        """The scene's hull buffer, record by record, at the same offsets (the scene packs from 0)."""
        offs = list(getattr(scene, 'hull_offsets', []))
        words = getattr(scene, 'hull_words', np.zeros(0, np.uint32))
        for k, at in enumerate(offs):
            end = offs[k + 1] if k + 1 < len(offs) else len(words) // 4
            rec = words[4 * at:4 * end].copy()
            for j in (0, 2, 4, 6):
                rec[j] -= at
            got = self.add_hull(rec)
            if got != at:
                raise AvbdError(_abi.AVBD_ERR_INVALID, f'hull record landed at {got}, the scene packed it at {at}')

    def add_bodies(self, records: np.ndarray) -> int:
        records = np.ascontiguousarray(records, dtype=BODY_DTYPE)
        first = ctypes.c_uint32()
        self._check(self.lib.avbd_add_bodies(self.handle, ptr(records), len(records), ctypes.byref(first)))
        return first.value

    def write_bodies(self, first: int, records: np.ndarray, keep_contacts: bool = False):
        records = np.ascontiguousarray(records, dtype=BODY_DTYPE)
        self._check(self.lib.avbd_write_bodies(self.handle, first, ptr(records), len(records), 1 if keep_contacts else 0))

    def write_bodies_at(self, indices, records: np.ndarray):
        """rewriteBodies(indices, bodies): any existing slots, each starting afresh."""
        i = np.ascontiguousarray(indices, dtype=np.uint32)
        records = np.ascontiguousarray(records, dtype=BODY_DTYPE)
        self._check(self.lib.avbd_write_bodies_at(self.handle, uptr(i), ptr(records), len(i)))

    def add_joints(self, records: np.ndarray, info: np.ndarray) -> int:
        records = np.ascontiguousarray(records, dtype=JOINT_DTYPE)
        info = np.ascontiguousarray(info, dtype=INFO_DTYPE)
        first = ctypes.c_uint32()
        self._check(self.lib.avbd_add_joints(self.handle, ptr(records), ptr(info), len(records), ctypes.byref(first)))
        return first.value

    def write_joints(self, first: int, records: np.ndarray, info: np.ndarray):
        records = np.ascontiguousarray(records, dtype=JOINT_DTYPE)
        info = np.ascontiguousarray(info, dtype=INFO_DTYPE)
        self._check(self.lib.avbd_write_joints(self.handle, first, ptr(records), ptr(info), len(records)))

    def append_joints(self, records: np.ndarray, info: np.ndarray) -> np.ndarray:
        """appendJoints / appendSprings: released slots first (lowest first), then new ones; the slots."""
        records = np.ascontiguousarray(records, dtype=JOINT_DTYPE)
        info = np.ascontiguousarray(info, dtype=INFO_DTYPE)
        slots = np.zeros(len(records), dtype=np.uint32)
        self._check(self.lib.avbd_append_joints(self.handle, ptr(records), ptr(info), len(records), uptr(slots)))
        return slots

    def release_joints(self, slots):
        """releaseJoints: the slots stop acting, their bodies collide again, the slots are reused."""
        s = np.ascontiguousarray(slots, dtype=np.uint32)
        self._check(self.lib.avbd_release_joints(self.handle, uptr(s), len(s)))

    def disable_joints(self, slots):
        """disableConstraint: penalties, stiffnesses and multipliers zeroed; the slots stay taken."""
        s = np.ascontiguousarray(slots, dtype=np.uint32)
        self._check(self.lib.avbd_disable_joints(self.handle, uptr(s), len(s)))

    def append_world_joint(self, body: int, anchor_world, anchor_body) -> int:
        """appendWorldJoint(b, anchorWorld, anchorBody), 'legacy' policy: holds the body's point
        `anchor_body` (body frame) at the world point `anchor_world`, free to turn; returns its slot."""
        aw = (ctypes.c_float * 3)(*[float(x) for x in anchor_world])
        ab = (ctypes.c_float * 3)(*[float(x) for x in anchor_body])
        slot = ctypes.c_uint32()
        self._check(self.lib.avbd_add_world_joint(self.handle, int(body), aw, ab, ctypes.byref(slot)))
        return slot.value

    def set_world_anchor(self, slot: int, p):
        """setWorldAnchor(slot, p): the joint's world point (r_a) from the next step on."""
        q = (ctypes.c_float * 3)(*[float(x) for x in p])
        self._check(self.lib.avbd_set_world_anchor(self.handle, int(slot), q))

    def body_storage(self) -> dict:
        """bodyBuffer: device addresses of the ten float4 field arrays (avbd_body record rows, in
        order), the bodies in use and the arrays' length."""
        v = _abi.BodyView()
        self._check(self.lib.avbd_body_storage(self.handle, ctypes.byref(v)))
        return {'fields': [int(f or 0) for f in v.fields], 'count': v.count, 'capacity': v.capacity}

    def contact_storage(self, which: int = 0) -> dict:
        """contactStorage (which 0: what the last step wrote) / contactStorages() (which 1: the step
        before's): device addresses of the pair words, normals and points, the counters and the word
        holding the pair-slot count, and the pair-slot capacity."""
        v = _abi.ContactView()
        self._check(self.lib.avbd_contact_storage(self.handle, int(which), ctypes.byref(v)))
        return {'pairs': int(v.pairs or 0), 'normals': int(v.normals or 0), 'points': int(v.points or 0), 'counters': int(v.counters or 0),
                'count_word': v.count_word, 'pair_capacity': v.pair_capacity}

    def add_ignore_pairs(self, pairs: np.ndarray):
        p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1, 2)
        self._check(self.lib.avbd_add_ignore_pairs(self.handle, uptr(p), len(p)))

    def set_filters_at(self, indices, groups, collides_with):
        """setFilters(indices, groups, collidesWith): any list of slots."""
        i = np.ascontiguousarray(indices, dtype=np.uint32)
        g = np.ascontiguousarray(np.asarray(groups, dtype=np.int64) & 0xFFFFFFFF, dtype=np.uint32)
        m = np.ascontiguousarray(np.asarray(collides_with, dtype=np.int64) & 0xFFFFFFFF, dtype=np.uint32)
        self._check(self.lib.avbd_set_filters_at(self.handle, uptr(i), uptr(g), uptr(m), len(i)))

    def set_filters(self, first: int, groups_mask: np.ndarray):
        g = np.ascontiguousarray(groups_mask, dtype=np.uint32).reshape(-1, 2)
        self._check(self.lib.avbd_set_filters(self.handle, first, uptr(g), len(g)))

    def set_body_aux(self, indices, scales, linear=None, angular=None):
        """setBodyAux: per-slot gravity scale and (both or neither) linear / angular damping rates."""
        idx = np.ascontiguousarray(indices, dtype=np.uint32)
        sc = np.ascontiguousarray(scales, dtype=np.float32)
        lin = None if linear is None else np.ascontiguousarray(linear, dtype=np.float32)
        ang = None if angular is None else np.ascontiguousarray(angular, dtype=np.float32)
        p = lambda a: a.ctypes.data if a is not None else None
        self._check(self.lib.avbd_set_body_aux(self.handle, p(idx), len(idx), p(sc), p(lin), p(ang)))

    def read_body_aux(self, first: int = 0, n: int | None = None) -> np.ndarray:
        n = self.body_count - first if n is None else n
        out = np.zeros((n, 4), np.float32)
        self._check(self.lib.avbd_read_body_aux(self.handle, first, out.ctypes.data, n))
        return out

    def set_lifecycle(self, index: int, bits: int):
        """setLifecycle: 2 disabled, 4 cold (joints start afresh); the slot loses its contact history."""
        self._check(self.lib.avbd_set_lifecycle(self.handle, index, bits))

    def seed_contacts(self, manifolds: np.ndarray, contacts: np.ndarray):
        m = np.ascontiguousarray(manifolds, dtype=MANIFOLD_DTYPE)
        c = np.ascontiguousarray(contacts, dtype=CONTACT_DTYPE)
        self._check(self.lib.avbd_seed_contacts(self.handle, ptr(m), len(m), ptr(c), len(c)))

    def set_fixed_colors(self, colors):
        if colors is None:
            self._check(self.lib.avbd_set_fixed_colors(self.handle, None, 0))
        else:
            c = np.ascontiguousarray(colors, dtype=np.uint32)
            self._check(self.lib.avbd_set_fixed_colors(self.handle, uptr(c), len(c)))
        self.fixed_colors = colors

    def sequential_colors(self) -> np.ndarray:
        """One colour per dynamic body, newest first: the reference's Gauss-Seidel order
        (GpuSolver3D.sequentialColors, solver.ts:1365-1372). At most 64 dynamic bodies."""
        b = self.read_bodies()
        colors = np.full(len(b), NO_COLOR, dtype=np.uint32)
        nxt = 0
        for i in range(len(b) - 1, -1, -1):
            if b[i]['mass'] > 0:
                colors[i] = nxt
                nxt += 1
        if nxt > _abi.MAX_COLORS:
            raise ValueError(f'sequential_colors: {nxt} dynamic bodies, at most {_abi.MAX_COLORS}')
        return colors

    # --- stepping ---
    def step(self, n: int = 1, reuse_manifolds: bool = False):
        """step(options) (gpu/solver.ts:2112): n steps; reuse_manifolds keeps last step's manifolds
        and detects no pair (substeps after a detecting step; applies while they are valid)."""
        if reuse_manifolds:
            opts = _abi.StepOptions(reuse_manifolds=1)
            self._check(self.lib.avbd_step_with(self.handle, n, ctypes.byref(opts)))
        else:
            self._check(self.lib.avbd_step(self.handle, n))

    # --- around the step: impulses, contact events, raycasts ---
    def apply_pushes(self, pushes: np.ndarray):
        """Pusher.apply (src/lib/push.ts:103-131): PUSH_DTYPE records (body, lin, off_lin, moment), one
        per body, applied to the velocities now, before the next step."""
        pushes = np.ascontiguousarray(pushes, dtype=_abi.PUSH_DTYPE)
        self._check(self.lib.avbd_apply_pushes(self.handle, ptr(pushes), len(pushes)))

    def contact_watch(self, pairs: int, capacity: int = 4096) -> 'ContactWatch':
        """A ContactWatch (src/lib/contacts.ts) on this world's contacts."""
        return ContactWatch(self, pairs, capacity)

    def pose_capture(self, max_frames: int, slots=None) -> 'PoseCapture':
        """A device recorder of pose cache frames (src/bake/pose-cache.ts) of `slots` (default: every body)."""
        return PoseCapture(self, max_frames, slots)

    def raycast(self, origins, directions, max_distance=None, ignore=(), mask: int = 0xFFFFFFFF) -> np.ndarray:
        """Raycaster.cast (src/lib/raycast.ts:170-251): the nearest hit of each ray (HIT_DTYPE; body -1: none)."""
        o = np.asarray(origins, dtype=np.float32).reshape(-1, 3)
        d = np.asarray(directions, dtype=np.float32).reshape(-1, 3)
        rays = np.zeros(len(o), dtype=_abi.RAY_DTYPE)
        rays['origin'] = o
        rays['direction'] = d
        rays['max_distance'] = 3.0e38 if max_distance is None else np.asarray(max_distance, dtype=np.float32)
        ig = np.ascontiguousarray(ignore, dtype=np.uint32)
        hits = np.zeros(len(o), dtype=_abi.HIT_DTYPE)
        self._check(self.lib.avbd_raycast(self.handle, ptr(rays), len(rays), uptr(ig) if ig.size else None, ig.size, mask, ptr(hits)))
        return hits

    def read_reuse_state(self) -> dict:
        """Contact-reuse state: reference poses (n, 8), moved steps (per body) and the generating step
        of each manifold (avbd_read_contacts' order)."""
        nb, nm = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self.lib.avbd_read_reuse_state(self.handle, None, 0, ctypes.byref(nb), None, 0, ctypes.byref(nm)))
        refs = np.zeros((max(nb.value, 1), 8), dtype=np.float32)
        gen = np.zeros(max(nm.value, 1), dtype=np.uint32)
        self._check(self.lib.avbd_read_reuse_state(self.handle, refs.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nb.value, ctypes.byref(nb),
                                                   uptr(gen), nm.value, ctypes.byref(nm)))
        moved = self.read_bodies()['moved_step'].view(np.uint32).copy()
        return {'refs': refs[:nb.value], 'moved': moved, 'generated': gen[:nm.value], 'step': self.read_counters()['steps']}

    def synchronize(self):
        self._check(self.lib.avbd_synchronize(self.handle))

    def use_graphs(self, on: bool = True):
        """Replay each step as a captured CUDA graph (default on)."""
        self._check(self.lib.avbd_use_graphs(self.handle, 1 if on else 0))

    def set_solve_blocks(self, blocks: int = 0):
        """Blocks of the cooperative topology + solve launch (0: all co-resident ones)."""
        self._check(self.lib.avbd_set_solve_blocks(self.handle, blocks))

    def enable_step_stats(self, capacity: int):
        """Record per-step device times and counters into a ring of `capacity` steps (no host syncs)."""
        self._check(self.lib.avbd_enable_step_stats(self.handle, capacity))

    def read_step_stats(self) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_read_step_stats(self.handle, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=_abi.STEP_STATS_DTYPE)
        self._check(self.lib.avbd_read_step_stats(self.handle, ptr(out), n.value, ctypes.byref(n)))
        return out

    def read_phase_clocks(self) -> np.ndarray:
        """Device time (ms) at each grid barrier of the last step's topology+solve launch."""
        out = np.zeros(1024, dtype=np.float64)
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_read_phase_clocks(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1024, ctypes.byref(n)))
        return out[:n.value]

    @property
    def stream(self) -> int:
        """The world's cudaStream_t, for torch.cuda.ExternalStream."""
        s = ctypes.c_void_p()
        self._check(self.lib.avbd_world_stream(self.handle, ctypes.byref(s)))
        return s.value or 0

    def write_bodies_async(self, records: np.ndarray, first: int = 0):
        """Pose/velocity upload from (pinned) host memory on the world's stream; shapes unchanged."""
        self._check(self.lib.avbd_write_bodies_async(self.handle, first, ptr(records), len(records)))

    # --- readbacks ---
    @property
    def body_count(self) -> int:
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_read_bodies(self.handle, None, 0, ctypes.byref(n)))
        return n.value

    def read_bodies(self) -> np.ndarray:
        n = self.body_count
        out = np.zeros(n, dtype=BODY_DTYPE)
        cnt = ctypes.c_uint32()
        self._check(self.lib.avbd_read_bodies(self.handle, ptr(out), n, ctypes.byref(cnt)))
        return out

    def read_bodies_into(self, out: np.ndarray, sync: bool = True):
        """Pose readback into caller memory (pinned for overlap), World.read's path."""
        self._check(self.lib.avbd_read_bodies_async(self.handle, ptr(out), len(out)))
        if sync:
            self.synchronize()

    def read_joints(self):
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_read_joints(self.handle, None, None, 0, ctypes.byref(n)))
        recs = np.zeros(n.value, dtype=JOINT_DTYPE)
        info = np.zeros(n.value, dtype=INFO_DTYPE)
        self._check(self.lib.avbd_read_joints(self.handle, ptr(recs), ptr(info), n.value, ctypes.byref(n)))
        return recs, info

    def read_counters(self) -> dict:
        c = Counters()
        self._check(self.lib.avbd_read_counters(self.handle, ctypes.byref(c)))
        return c.as_dict()

    def read_contacts(self):
        nm, nc = ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self.lib.avbd_read_contacts(self.handle, None, 0, ctypes.byref(nm), None, 0, ctypes.byref(nc)))
        m = np.zeros(nm.value, dtype=MANIFOLD_DTYPE)
        c = np.zeros(nc.value, dtype=CONTACT_DTYPE)
        self._check(self.lib.avbd_read_contacts(self.handle, ptr(m), nm.value, ctypes.byref(nm), ptr(c), nc.value, ctypes.byref(nc)))
        return m, c

    def read_contact_list(self) -> list[dict]:
        """readContactList (solver.ts:2311-2346): every point with its pair's bodies and normal."""
        m, c = self.read_contacts()
        out = []
        for rec in m:
            for k in range(int(rec['first']), int(rec['first'] + rec['count'])):
                key = int(c[k]['key'])
                out.append({'a': int(rec['a']), 'b': int(rec['b']), 'feature': key & ~_abi.STICK_BIT, 'stick': bool(key & _abi.STICK_BIT),
                            'rA': c[k]['r_a'].astype(np.float64), 'rB': c[k]['r_b'].astype(np.float64), 'pen': c[k]['pen'].astype(np.float64),
                            'lam': c[k]['lam'].astype(np.float64), 'normal': rec['normal'].astype(np.float64)})
        return out

    def read_pairs(self) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_read_pairs(self.handle, None, 0, ctypes.byref(n)))
        out = np.zeros(2 * n.value, dtype=np.uint32)
        self._check(self.lib.avbd_read_pairs(self.handle, uptr(out), n.value, ctypes.byref(n)))
        return out.reshape(-1, 2)

    def read_colors(self) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_read_colors(self.handle, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=np.uint32)
        self._check(self.lib.avbd_read_colors(self.handle, uptr(out), n.value, ctypes.byref(n)))
        return out


class PoseCapture:
    """Pose cache frames (src/bake/pose-cache.ts) gathered on the device (avbd_pose_capture_*): frame()
    after a step enqueues one gather of the slots' positions and rotations with the world's step word,
    without synchronising; read() returns them; to_pose_cache() makes the cache the codec writes."""

    def __init__(self, world: 'CudaSolver3D', max_frames: int, slots=None):
        self.world = world
        self.lib = world.lib
        n = world.body_count if slots is None else len(slots)
        self.slots = np.arange(n, dtype=np.uint32) if slots is None else np.ascontiguousarray(slots, dtype=np.uint32)
        self.max_frames = int(max_frames)
        h = ctypes.c_void_p()
        world._check(self.lib.avbd_pose_capture_create(world.handle, uptr(self.slots), len(self.slots), self.max_frames, ctypes.byref(h)))
        self.handle = h

    def frame(self):
        self.world._check(self.lib.avbd_pose_capture_frame(self.handle))

    def reset(self):
        self.world._check(self.lib.avbd_pose_capture_reset(self.handle))

    def read(self):
        """(steps uint32 [frames], poses float32 [frames, slots, 7], dropped)."""
        steps = np.zeros(self.max_frames, np.uint32)
        poses = np.zeros((self.max_frames, len(self.slots), 7), np.float32)
        n, dropped = ctypes.c_uint32(), ctypes.c_uint32()
        self.world._check(self.lib.avbd_pose_capture_read(self.handle, uptr(steps), poses.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                          self.max_frames, ctypes.byref(n), ctypes.byref(dropped)))
        return steps[:n.value], poses[:n.value], dropped.value

    def to_pose_cache(self, cache_id: int, ids=None, termination: str = 'complete', provenance=None):
        """The frames as a pose_cache.PoseCache: a body's id (default slot + 1), its shape (boxes and
        spheres; the cache holds nothing else), full size and fixed flag from its record, and its lifetime
        from the frames where its slot is not +0 (one run of frames per id)."""
        from . import pose_cache as pc
        steps, poses, _ = self.read()
        if len(steps) == 0:
            raise pc.PoseCacheError('data', 'a cache needs at least one frame')
        recs = self.world.read_bodies()[self.slots]
        ids = (self.slots.astype(np.int64) + 1) if ids is None else np.asarray(ids, dtype=np.int64)
        bodies = []
        for k, r in enumerate(recs):
            shape = int(r['shape'])
            if shape not in (0, 1):
                raise pc.PoseCacheError('data', f'slot {int(self.slots[k])}: the pose cache holds boxes and spheres only')
            alive = np.flatnonzero(np.any(poses[:, k].view(np.uint32) != 0, axis=1))
            if len(alive) == 0:
                raise pc.PoseCacheError('data', f'slot {int(self.slots[k])} is alive in no frame')
            first, end = int(alive[0]), int(alive[-1]) + 1
            size = [float(x) for x in r['size']]
            bodies.append(pc.PoseCacheBody(int(ids[k]), 'box' if shape == 0 else 'sphere', size, bool(r['mass'] <= 0), first, end))
        return pc.PoseCache(int(cache_id), float(self.world.params.dt), bodies, steps.copy(), poses.copy(), termination, provenance)

    def destroy(self):
        if getattr(self, 'handle', None):
            self.lib.avbd_pose_capture_destroy(self.handle)
            self.handle = None


class ContactWatch:
    """ContactWatch (src/lib/contacts.ts:129-267) over the C ABI: begin and end events of the touching
    pairs that have a reporting body, by lifetime IDs. Run it after each step; read drains the events."""

    def __init__(self, world: CudaSolver3D, pairs: int, capacity: int = 4096):
        self.world = world
        self.lib = world.lib
        h = ctypes.c_void_p()
        world._check(self.lib.avbd_contact_watch_create(world.handle, pairs, capacity, ctypes.byref(h)))
        self.handle = h
        self.capacity = capacity

    def _check(self, code: int):
        if code != _abi.AVBD_OK:
            msg = self.lib.avbd_contact_watch_last_error(self.handle)
            raise _abi.error(code, msg.decode() if msg else 'contact watch error')

    def set_watched(self, indices, ids, on):
        i = np.ascontiguousarray(indices, dtype=np.uint32)
        d = np.ascontiguousarray(ids, dtype=np.uint32)
        o = np.ascontiguousarray(np.asarray(on, dtype=bool).astype(np.uint32))
        if not (len(i) == len(d) == len(o)):
            raise _abi.error(_abi.AVBD_ERR_INVALID, 'set_watched: indices, ids and on differ in length')
        self._check(self.lib.avbd_contact_watch_set(self.handle, uptr(i), uptr(d), uptr(o), len(i)))

    def run(self, step: int, dt: float):
        self._check(self.lib.avbd_contact_watch_run(self.handle, step, dt))

    def read(self):
        """(events EVENT_DTYPE in step order, dropped, full)."""
        out = np.zeros(self.capacity, dtype=_abi.EVENT_DTYPE)
        n, dropped, full = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        self._check(self.lib.avbd_contact_watch_read(self.handle, ptr(out), self.capacity, ctypes.byref(n), ctypes.byref(dropped), ctypes.byref(full)))
        return out[:n.value], dropped.value, bool(full.value)

    def destroy(self):
        if getattr(self, 'handle', None):
            self.lib.avbd_contact_watch_destroy(self.handle)
            self.handle = None


def find_pairs_noalloc(bodies: np.ndarray, groups_mask: np.ndarray | None = None, cap: int = _abi.NOALLOC_MAX_PAIRS,
                       stream: int = 0) -> np.ndarray:
    """The step's candidate pairs of up to 4096 bodies (host records) through avbd_find_pairs_noalloc,
    which allocates nothing: its scratch is one fixed device array shared by every call, so calls must
    not overlap on the GPU. Returns an (k, 2) array of (a, b), a > b, in no particular order."""
    lib = _abi.load()
    bodies = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
    if len(bodies) > _abi.NOALLOC_MAX_BODIES:
        raise _abi.error(_abi.AVBD_ERR_CAPACITY, f'avbd_find_pairs_noalloc takes at most {_abi.NOALLOC_MAX_BODIES} bodies, got {len(bodies)}')
    gm = None if groups_mask is None else np.ascontiguousarray(groups_mask, dtype=np.uint32).reshape(-1)
    if gm is not None and gm.size != 2 * len(bodies):
        raise _abi.error(_abi.AVBD_ERR_INVALID, f'groups_mask holds {gm.size} words; (groups, mask) of {len(bodies)} bodies is {2 * len(bodies)}')
    out = np.zeros(2 * max(cap, 1), dtype=np.uint32)
    count = ctypes.c_uint32()
    code = lib.avbd_find_pairs_noalloc(ptr(bodies), len(bodies), uptr(gm) if gm is not None else None, uptr(out), cap, ctypes.byref(count),
                                       ctypes.c_void_p(stream))
    if code != _abi.AVBD_OK:
        if code == _abi.AVBD_ERR_CAPACITY:
            raise _abi.error(code, f'{count.value} pairs found, more than the {min(cap, _abi.NOALLOC_MAX_PAIRS)} that fit')
        raise _abi.error(code, 'avbd_find_pairs_noalloc failed')
    return out[:2 * count.value].reshape(-1, 2)


def device_info(device: int = 0):
    lib = _abi.load()
    name = ctypes.create_string_buffer(256)
    sms = ctypes.c_int()
    code = lib.avbd_device_info(device, name, 256, ctypes.byref(sms))
    if code != _abi.AVBD_OK:
        return None
    return name.value.decode(), sms.value
