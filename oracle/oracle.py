"""ctypes binding of the CPU oracle (avbd_oracle.cpp). TEST INFRASTRUCTURE: imported only by
tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, never by the product."""

from __future__ import annotations

import ctypes
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from build_oracle import build  # noqa: E402

_lib = None

BODY_REC = 43
FORCE_REC = 47
K_MANIFOLD, K_JOINT, K_SPRING, K_IGNORE = 0, 1, 2, 3
NO_COLOR = 255
PENDING = 256


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, '_build', 'liboracle.so')
        if not os.path.exists(path):
            path = build()
        L = ctypes.CDLL(path)
        P, D, I, U = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_uint
        L.orc_create.restype = P
        L.orc_create.argtypes = [I]
        L.orc_destroy.argtypes = [P]
        L.orc_set_params.argtypes = [P, D, U]
        L.orc_set_wind.argtypes = [P, D]
        L.orc_add_body.argtypes = [P, D]
        L.orc_body_count.argtypes = [P]
        L.orc_get_body.argtypes = [P, I, D]
        L.orc_set_body.argtypes = [P, I, D]
        L.orc_add_joint.argtypes = [P, I, I, D, D, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_add_spring.argtypes = [P, I, I, D, D, ctypes.c_double, ctypes.c_double]
        L.orc_add_ignore.argtypes = [P, I, I]
        L.orc_force_count.argtypes = [P]
        L.orc_get_force.argtypes = [P, I, D]
        L.orc_set_joint.argtypes = [P, I, D]
        L.orc_set_joint_anchor.argtypes = [P, I, D]
        L.orc_manifold_count.argtypes = [P]
        L.orc_contact_count.argtypes = [P]
        L.orc_get_manifolds.argtypes = [P, D, D]
        L.orc_set_contact_penalty.argtypes = [P, ctypes.c_double]
        L.orc_round_f32.argtypes = [P]
        L.orc_step_gpu_reuse.argtypes = [P, ctypes.POINTER(U), ctypes.POINTER(I)]
        F, PU = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(U)
        L.orc_get_reuse.argtypes = [P, PU, F, PU, PU]
        L.orc_set_reuse.argtypes = [P, U, F, PU, PU]
        L.orc_set_manifolds.argtypes = [P, I, D, I, D]
        L.orc_step.argtypes = [P]
        L.orc_step_gpu.argtypes = [P, ctypes.POINTER(U), ctypes.POINTER(I)]
        L.orc_pairs.argtypes = [P, ctypes.POINTER(U), I]
        L.orc_pairs.restype = I
        L.orc_narrowphase.argtypes = [P, I, I, I, D, D]
        L.orc_narrowphase.restype = I
        L.orc_color_graph.argtypes = [I, ctypes.POINTER(ctypes.c_ubyte), ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(U), I, I, ctypes.POINTER(I)]
        L.orc_set_threads.argtypes = [I]
        L.orc_set_threads.restype = I
        L.orc_hash32.argtypes = [U]
        L.orc_hash32.restype = U
        L.orc_set_hulls.argtypes = [P, ctypes.POINTER(U), I]
        L.orc_set_body_aux.argtypes = [P, I, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_set_lifecycle.argtypes = [P, I, U]
        L.orc_adj_record.argtypes = [P, I]
        L.orc_adj_record.restype = P
        L.orc_adj_destroy.argtypes = [P]
        L.orc_adj_bodies.argtypes = [P]
        L.orc_adj_bodies.restype = I
        L.orc_adj_points.argtypes = [P, I]
        L.orc_adj_points.restype = I
        L.orc_adj_nominal.argtypes = [P, D]
        L.orc_adj_set_target.argtypes = [P, D]
        L.orc_adj_loss.argtypes = [P, D, D]
        L.orc_adj_loss.restype = ctypes.c_double
        L.orc_adj_gradient.argtypes = [P, D, D]
        L.orc_adj_gradient.restype = ctypes.c_double
        L.orc_adj_sizes.argtypes = [P, ctypes.POINTER(I)]
        L.orc_adj_export.argtypes = [P, D] + [ctypes.POINTER(I)] * 3 + [D, D] + [ctypes.POINTER(I)] * 4
        L.orc_adj_import.argtypes = [D, I, I, D, D] + [ctypes.POINTER(I)] * 3 + [D, D] + [ctypes.POINTER(I)] * 4
        L.orc_adj_import.restype = P
        L.orc_adj_param.argtypes = [P, I]
        L.orc_adj_param.restype = ctypes.c_double
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def body_record(b) -> np.ndarray:
    r = np.zeros(BODY_REC)
    r[0:3] = b.pos
    r[3:7] = b.rot
    r[7:10] = b.vel
    r[10:13] = b.ang_vel
    r[13:16] = b.prev_vel
    r[16:19] = b.size
    r[19] = b.mass
    r[20:23] = b.moment
    r[23] = b.friction
    r[24] = b.radius
    r[25] = b.shape
    r[26:29] = b.initial_pos
    r[29:33] = b.initial_rot
    r[33:36] = b.inertial_pos
    r[36:40] = b.inertial_rot
    r[40] = b.groups
    r[41] = b.mask
    r[42] = NO_COLOR
    return r


STICK_BIT = 0x80000000


def records_from_cuda_bodies(bodies: np.ndarray, colors: np.ndarray, base: np.ndarray) -> np.ndarray:
    """Oracle body records (doubles) holding CUDA body records (the C ABI's avbd_body fields) and colour
    state; `base` (oracle records of the same bodies) supplies what a CUDA record does not hold (the
    collision filters)."""
    r = np.array(base, dtype=np.float64, copy=True)
    r[:, 0:3] = bodies['pos']
    r[:, 3:7] = bodies['rot']
    r[:, 7:10] = bodies['vel']
    r[:, 10:13] = bodies['ang_vel']
    r[:, 13:15] = 0.0
    r[:, 15] = bodies['prev_up_vel']  # up = +z: only this component is read
    r[:, 16:19] = bodies['size']
    r[:, 19] = bodies['mass']
    r[:, 20:23] = bodies['moment']
    r[:, 23] = bodies['friction']
    r[:, 24] = bodies['radius']
    r[:, 25] = bodies['shape']
    r[:, 26:29] = bodies['initial_pos']
    r[:, 29:33] = bodies['initial_rot']
    r[:, 33:36] = bodies['inertial_pos']
    r[:, 36:40] = bodies['inertial_rot']
    r[:, 42] = colors
    return r


def records_from_cuda_contacts(m: np.ndarray, c: np.ndarray):
    """CUDA manifolds and contacts (avbd_read_contacts: manifold.first indexes the contacts) in the
    layout of Oracle.manifolds() / Oracle.set_manifolds()."""
    mrec = np.zeros((len(m), 8))
    mrec[:, 1] = m['a']
    mrec[:, 2] = m['b']
    mrec[:, 3] = m['count']
    mrec[:, 4:7] = m['normal']
    mrec[:, 7] = m['friction']
    if len(m):
        first = m['first'].astype(np.int64)
        count = m['count'].astype(np.int64)
        idx = np.repeat(first - np.concatenate([[0], np.cumsum(count)[:-1]]), count) + np.arange(int(count.sum()))
    else:
        idx = np.zeros(0, np.int64)
    q = c[idx]
    crec = np.zeros((len(q), 17))
    crec[:, 0] = q['key'] & np.uint32(~STICK_BIT & 0xFFFFFFFF)
    crec[:, 1] = (q['key'] & np.uint32(STICK_BIT)) != 0
    crec[:, 2:5] = q['r_a']
    crec[:, 5:8] = q['r_b']
    crec[:, 8] = q['c0_n']
    crec[:, 9] = q['c0_t1']
    crec[:, 10] = q['c0_t2']
    crec[:, 11:14] = q['pen']
    crec[:, 14:17] = q['lam']
    return mrec, crec


class Oracle:
    """One CPU solver instance (fp32=False: double, the reference's precision)."""

    def __init__(self, scene=None, fp32: bool = False, flags: int = 0):
        self.L = lib()
        self.h = self.L.orc_create(1 if fp32 else 0)
        self.fp32 = fp32
        self.force_of = []  # scene force index -> oracle force index
        if scene is not None:
            self.load(scene, flags)

    def __del__(self):
        if getattr(self, 'h', None):
            self.L.orc_destroy(self.h)
            self.h = None

    def set_params(self, p, flags: int = 0):
        arr = np.array([p.dt, p.gravity, p.iterations, p.alpha, p.beta_lin, p.beta_ang, p.gamma, p.contact_margin], dtype=np.float64)
        self.L.orc_set_params(self.h, _dp(arr), flags)
        self.set_wind(getattr(p, 'wind_speed', 0.0), getattr(p, 'wind_angle', 0.0), getattr(p, 'wind_gust', 0.4), getattr(p, 'wind_pressure', 0.0))

    def set_wind(self, speed: float, angle: float, gust: float = 0.4, pressure: float = 0.72):
        """The wind on sails (GPU mode): speed (m/s) towards angle (rad from +x about z), gusts, pressure
        coefficient 1/2 rho C_d; its velocity in f32 as the device's parameters hold it
        (gpu/solver.ts:1994-1998)."""
        wx = float(np.float32(speed * np.cos(angle)))
        wy = float(np.float32(speed * np.sin(angle)))
        arr = np.array([wx, wy, float(np.float32(gust)), float(np.float32(pressure))], dtype=np.float64)
        self.L.orc_set_wind(self.h, _dp(arr))

    def set_body_aux(self, i: int, scale: float, linear: float = 0.0, angular: float = 0.0):
        """GPU-mode aux record of body i: gravity scale and damping rates (1/s)."""
        self.L.orc_set_body_aux(self.h, i, scale, linear, angular)

    def set_lifecycle(self, i: int, bits: int):
        """GPU-mode lifecycle bits of body i (4: cold, its joints start the next step afresh)."""
        self.L.orc_set_lifecycle(self.h, i, bits)

    def set_hulls(self, words):
        """The hull buffer the bodies' shape codes name (gpu/solver.ts:313-338 layout)."""
        w = np.ascontiguousarray(words, dtype=np.uint32)
        self._hulls = w
        self.L.orc_set_hulls(self.h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), len(w))

    def load(self, scene, flags: int = 0):
        self.set_params(scene.params, flags)
        if len(getattr(scene, 'hull_words', [])):
            self.set_hulls(scene.hull_words)
        for b in scene.bodies:
            self.L.orc_add_body(self.h, _dp(body_record(b)))
        for f in scene.forces:
            rA = np.array(f.rA, dtype=np.float64)
            rB = np.array(f.rB, dtype=np.float64)
            if f.kind == 'joint':
                k = self.L.orc_add_joint(self.h, f.a, f.b, _dp(rA), _dp(rB), f.stiffness_lin, f.stiffness_ang, f.fracture)
                rec = self.force(k)
                rec[24] = 1.0 if f.fracture_linear else 0.0
                rec[27] = f.yield_force
                rec[28] = f.break_bend
                if f.rest is not None:
                    rec[29:33] = f.rest
                    rec[33] = 1
                if f.rest_start is not None:
                    rec[34:38] = f.rest_start
                    rec[38] = 1
                rec[3:6] = f.penalty_lin
                rec[6:9] = f.penalty_ang
                self.set_joint(k, rec)
            elif f.kind == 'spring':
                k = self.L.orc_add_spring(self.h, f.a, f.b, _dp(rA), _dp(rB), f.spring_stiffness, f.spring_rest)
            else:
                k = self.L.orc_add_ignore(self.h, f.a, f.b)
            self.force_of.append(k)

    # --- state ---
    @property
    def body_count(self):
        return self.L.orc_body_count(self.h)

    def _body_index(self, i):
        if not 0 <= i < self.body_count:
            raise IndexError(f'body {i} of {self.body_count}')

    def _joint_index(self, i):
        if not 0 <= i < self.force_count or int(self.force(i)[0]) != K_JOINT:
            raise IndexError(f'force {i} is not a joint')

    def body(self, i) -> np.ndarray:
        self._body_index(i)
        r = np.zeros(BODY_REC)
        self.L.orc_get_body(self.h, i, _dp(r))
        return r

    def bodies(self) -> np.ndarray:
        return np.stack([self.body(i) for i in range(self.body_count)]) if self.body_count else np.zeros((0, BODY_REC))

    def set_body(self, i, rec):
        self._body_index(i)
        rec = np.ascontiguousarray(rec, dtype=np.float64)
        self.L.orc_set_body(self.h, i, _dp(rec))

    @property
    def force_count(self):
        return self.L.orc_force_count(self.h)

    def force(self, i) -> np.ndarray:
        if not 0 <= i < self.force_count:
            raise IndexError(f'force {i} of {self.force_count}')
        r = np.zeros(FORCE_REC)
        self.L.orc_get_force(self.h, i, _dp(r))
        return r

    def set_joint(self, i, rec):
        self._joint_index(i)
        rec = np.ascontiguousarray(rec, dtype=np.float64)
        self.L.orc_set_joint(self.h, i, _dp(rec))

    def set_joint_anchor(self, i, p):
        """setWorldAnchor: joint i's rA (its world point when it has no body A)."""
        self._joint_index(i)
        q = np.ascontiguousarray(p, dtype=np.float64)
        self.L.orc_set_joint_anchor(self.h, i, _dp(q))

    def manifolds(self):
        nm = self.L.orc_manifold_count(self.h)
        nc = self.L.orc_contact_count(self.h)
        m = np.zeros((max(nm, 1), 8))
        c = np.zeros((max(nc, 1), 17))
        self.L.orc_get_manifolds(self.h, _dp(m), _dp(c))
        return m[:nm], c[:nc]

    def set_contact_penalty(self, pen):
        self.L.orc_set_contact_penalty(self.h, pen)

    def round_f32(self):
        """Rounds every state value to f32 in place: the state a CUDA world seeded from this one holds."""
        self.L.orc_round_f32(self.h)

    def set_bodies(self, recs: np.ndarray):
        """Overwrites bodies 0 .. len(recs) - 1 with oracle body records."""
        recs = np.ascontiguousarray(recs, dtype=np.float64)
        for i in range(len(recs)):
            self.set_body(i, recs[i])

    def load_cuda_state(self, bodies: np.ndarray, colors: np.ndarray, manifolds: np.ndarray, contacts: np.ndarray):
        """The bodies, colour state and last step's contacts of a CUDA world (C-ABI records) that holds
        this oracle's bodies in the same order: both then start the next step from the same values."""
        self.set_bodies(records_from_cuda_bodies(bodies, colors[:len(bodies)], self.bodies()))
        self.set_manifolds(*records_from_cuda_contacts(manifolds, contacts))

    def set_manifolds(self, m: np.ndarray, c: np.ndarray):
        """Replaces last step's manifolds (manifolds()' layout: 8 per manifold, 17 per contact)."""
        m = np.ascontiguousarray(m, dtype=np.float64).reshape(-1, 8)
        c = np.ascontiguousarray(c, dtype=np.float64).reshape(-1, 17)
        mm = m if len(m) else np.zeros((1, 8))
        cc = c if len(c) else np.zeros((1, 17))
        self.L.orc_set_manifolds(self.h, len(m), _dp(mm), len(c), _dp(cc))

    # --- stepping ---
    def step(self, n: int = 1):
        for _ in range(n):
            self.L.orc_step(self.h)

    def step_gpu(self, fixed_colors=None, reuse_manifolds: bool = False):
        """One GPU-mode step; reuse_manifolds: keep every manifold of last step, detect no pair (the
        step option reuseManifolds)."""
        stats = (ctypes.c_int * 3)()
        fn = self.L.orc_step_gpu_reuse if reuse_manifolds else self.L.orc_step_gpu
        if fixed_colors is None:
            fn(self.h, None, stats)
        else:
            fc = np.ascontiguousarray(fixed_colors, dtype=np.uint32)
            fn(self.h, fc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), stats)
        return {'colors': stats[0], 'clashes': stats[1], 'rounds': stats[2]}

    def reuse_state(self) -> dict:
        """Contact-reuse state: step counter, reference poses (n, 8), moved steps, manifold generations."""
        n = self.body_count
        nm = self.L.orc_manifold_count(self.h)
        step = ctypes.c_uint()
        refs = np.zeros((max(n, 1), 8), dtype=np.float32)
        moved = np.zeros(max(n, 1), dtype=np.uint32)
        gen = np.zeros(max(nm, 1), dtype=np.uint32)
        F, PU = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint)
        self.L.orc_get_reuse(self.h, ctypes.byref(step), refs.ctypes.data_as(F), moved.ctypes.data_as(PU), gen.ctypes.data_as(PU))
        return {'step': step.value, 'refs': refs[:n], 'moved': moved[:n], 'generated': gen[:nm]}

    def set_reuse_state(self, step: int, refs, moved, generated):
        F, PU = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint)
        refs = np.ascontiguousarray(refs, dtype=np.float32).reshape(-1, 8)
        moved = np.ascontiguousarray(moved, dtype=np.uint32)
        gen = np.ascontiguousarray(generated, dtype=np.uint32)
        self.L.orc_set_reuse(self.h, int(step), refs.ctypes.data_as(F), moved.ctypes.data_as(PU), gen.ctypes.data_as(PU) if gen.size else None)

    def pairs(self) -> np.ndarray:
        cap = 1 << 16
        while True:
            out = np.zeros(2 * cap, dtype=np.uint32)
            n = self.L.orc_pairs(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), cap)
            if n <= cap:
                return out[: 2 * n].reshape(-1, 2)
            cap = n

    def narrowphase(self, a, b, face_bias=False):
        out = np.zeros(8 * 7)
        normal = np.zeros(3)
        n = self.L.orc_narrowphase(self.h, a, b, 1 if face_bias else 0, _dp(out), _dp(normal))
        rows = out[: 7 * n].reshape(-1, 7)
        return [(int(r[0]), r[1:4].copy(), r[4:7].copy()) for r in rows], normal

    def colors(self) -> np.ndarray:
        return self.bodies()[:, 42].astype(np.uint32)

    def adjoint(self, steps: int) -> 'Adjoint':
        return Adjoint(self, steps)


def set_threads(n: int) -> int:
    """OpenMP threads of the GPU-mode step (0: keep); returns the count in use."""
    return lib().orc_set_threads(n)


def sequential_colors(scene) -> np.ndarray:
    """One colour per dynamic body, newest first: the reference's Gauss-Seidel order
    (gpu/solver.ts:1365-1372)."""
    colors = np.full(len(scene.bodies), NO_COLOR, dtype=np.uint32)
    nxt = 0
    for i in range(len(scene.bodies) - 1, -1, -1):
        if scene.bodies[i].mass > 0:
            colors[i] = nxt
            nxt += 1
    assert nxt <= 64, f'{nxt} dynamic bodies, at most 64'
    return colors


def color_graph(n, dynamic, start, nbr, state, cap=64, max_rounds=64):
    L = lib()
    dyn = np.ascontiguousarray(dynamic, dtype=np.uint8)
    st = np.ascontiguousarray(start, dtype=np.int32)
    nb = np.ascontiguousarray(nbr, dtype=np.int32) if len(nbr) else np.zeros(1, dtype=np.int32)
    s = np.ascontiguousarray(state, dtype=np.uint32).copy()
    stats = (ctypes.c_int * 3)()
    L.orc_color_graph(n, dyn.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                      nb.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), s.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), cap, max_rounds, stats)
    return s, {'colors': stats[0], 'clashes': stats[1], 'rounds': stats[2]}


class Adjoint:
    """The FP64 adjoint of the GPU-mode step with the contact structure frozen: `Oracle.adjoint(steps)`
    records that many steps of the oracle's scene (advancing it); `loss`/`gradient` replay them with
    any parameters (8 per body: v0, omega0, mass, friction)."""

    def __init__(self, oracle: 'Oracle', steps: int):
        self.L = oracle.L
        self.h = self.L.orc_adj_record(oracle.h, steps)
        if not self.h:
            raise ValueError('adjoint problems need the FP64 oracle and a scene without joints')
        self.n = self.L.orc_adj_bodies(self.h)
        self.steps = steps

    @classmethod
    def from_record(cls, rec: dict, nominal: np.ndarray) -> 'Adjoint':
        """A problem from one world's recorded structure in the export() layout (for instance the
        GPU recording's world, split out) with its nominal parameters (8 per body)."""
        self = cls.__new__(cls)
        self.L = lib()
        P = rec['params']
        p7 = np.array([P['dt'], P['gravity'], P['alpha'], P['gamma'], P['beta_lin'], P['contact_margin'], P['iterations']], np.float64)
        keep = [np.ascontiguousarray(rec[k], np.int32) for k in ('step_man', 'step_pt', 'man_bodies', 'pt_man', 'pt_prev', 'colors', 'ncol')]
        dk = [np.ascontiguousarray(x, np.float64) for x in (rec['bodies'], nominal, rec['basis'], rec['anchors'])]
        I = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        self.h = self.L.orc_adj_import(_dp(p7), int(rec['n']), int(rec['steps']), _dp(dk[0]), _dp(dk[1]), I(keep[0]), I(keep[1]), I(keep[2]),
                                       _dp(dk[2]), _dp(dk[3]), I(keep[3]), I(keep[4]), I(keep[5]), I(keep[6]))
        self.n = int(rec['n'])
        self.steps = int(rec['steps'])
        return self

    def __del__(self):
        if getattr(self, 'h', None):
            self.L.orc_adj_destroy(self.h)
            self.h = None

    def nominal(self) -> np.ndarray:
        out = np.zeros(8 * self.n)
        self.L.orc_adj_nominal(self.h, _dp(out))
        return out

    def set_target(self, target: np.ndarray):
        t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
        self.L.orc_adj_set_target(self.h, _dp(t))

    def loss(self, params: np.ndarray, final: bool = False):
        p = np.ascontiguousarray(params, dtype=np.float64)
        out = np.zeros(7 * self.n)
        L = self.L.orc_adj_loss(self.h, _dp(p), _dp(out))
        return (L, out.reshape(-1, 7)) if final else L

    def export(self) -> dict:
        """The recorded structure as flat arrays (indices over all steps of this one world)."""
        ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        sz = np.zeros(2, dtype=np.int32)
        self.L.orc_adj_sizes(self.h, ip(sz))
        nm, npts, n, K = int(sz[0]), int(sz[1]), self.n, self.steps
        out = {'bodies': np.zeros(13 * n), 'step_man': np.zeros(K + 1, np.int32), 'step_pt': np.zeros(K + 1, np.int32),
               'man_bodies': np.zeros(2 * max(nm, 1), np.int32), 'basis': np.zeros(9 * max(nm, 1)), 'anchors': np.zeros(6 * max(npts, 1)),
               'pt_man': np.zeros(max(npts, 1), np.int32), 'pt_prev': np.zeros(max(npts, 1), np.int32), 'colors': np.zeros(K * n, np.int32),
               'ncol': np.zeros(K, np.int32)}
        self.L.orc_adj_export(self.h, _dp(out['bodies']), ip(out['step_man']), ip(out['step_pt']), ip(out['man_bodies']), _dp(out['basis']),
                              _dp(out['anchors']), ip(out['pt_man']), ip(out['pt_prev']), ip(out['colors']), ip(out['ncol']))
        out['params'] = {k: self.L.orc_adj_param(self.h, i) for i, k in enumerate(['dt', 'gravity', 'alpha', 'gamma', 'beta_lin', 'contact_margin',
                                                                                     'iterations'])}
        out['n'], out['steps'], out['manifolds'], out['points'] = n, K, nm, npts
        return out

    def gradient(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float64)
        g = np.zeros(8 * self.n)
        L = self.L.orc_adj_gradient(self.h, _dp(p), _dp(g))
        return L, g
