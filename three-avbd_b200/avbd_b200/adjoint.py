"""The adjoint of the step (avbd_adjoint_* in include/avbd.h): gradients of a final-pose loss with
respect to every body's initial velocities, mass and friction, for batched worlds, with the contact
structure frozen from a recorded rollout.

A recording is one world's structure as flat arrays (`bodies` 13 per body; per step its manifolds
with their bases and points with their anchors and warm-start source; the colouring); `Adjoint`
takes a list of them, one per world.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _abi


class AdjointDesc(ctypes.Structure):
    _fields_ = [('worlds', ctypes.c_uint32), ('steps', ctypes.c_uint32), ('iterations', ctypes.c_uint32), ('checkpoint', ctypes.c_uint32),
                ('dt', ctypes.c_double), ('gravity', ctypes.c_double), ('alpha', ctypes.c_double), ('gamma', ctypes.c_double),
                ('beta_lin', ctypes.c_double), ('contact_margin', ctypes.c_double)] + \
               [(n, ctypes.c_void_p) for n in ('world_first_body', 'bodies', 'step_first_manifold', 'step_first_point', 'manifold_bodies',
                                               'manifold_basis', 'point_anchors', 'point_manifold', 'point_prev', 'colors', 'color_counts')] + \
               [('device', ctypes.c_int32)]


def combine(records: list) -> dict:
    """World recordings (indices over their own steps) as one batch, step-major: step s holds every
    world's manifolds and points of that step, world by world."""
    W, K = len(records), records[0]['steps']
    assert all(r['steps'] == K for r in records)
    nbs = [r['n'] for r in records]
    first_body = np.concatenate([[0], np.cumsum(nbs)]).astype(np.uint32)
    bodies = np.concatenate([r['bodies'] for r in records])
    step_man = np.zeros(K * (W + 1), np.uint32)
    step_pt = np.zeros(K * (W + 1), np.uint32)
    mb, basis, anchors, pt_man, pt_prev = [], [], [], [], []
    m = p = 0
    gpt = {}  # (world, step, local point) -> global point
    for s in range(K):
        for w, r in enumerate(records):
            step_man[s * (W + 1) + w] = m
            step_pt[s * (W + 1) + w] = p
            m0, m1 = int(r['step_man'][s]), int(r['step_man'][s + 1])
            p0, p1 = int(r['step_pt'][s]), int(r['step_pt'][s + 1])
            mb.append(r['man_bodies'][2 * m0:2 * m1])
            basis.append(r['basis'][9 * m0:9 * m1])
            anchors.append(r['anchors'][6 * p0:6 * p1])
            pt_man.append(r['pt_man'][p0:p1] - m0 + m)
            prev = r['pt_prev'][p0:p1].copy()
            if s > 0:
                q0 = int(r['step_pt'][s - 1])
                base = gpt[(w, s - 1)]
                prev = np.where(prev >= 0, prev - q0 + base, -1)
            pt_prev.append(prev)
            gpt[(w, s)] = p
            m += m1 - m0
            p += p1 - p0
        step_man[s * (W + 1) + W] = m
        step_pt[s * (W + 1) + W] = p
    colors = np.concatenate([np.concatenate([r['colors'][s * r['n']:(s + 1) * r['n']] for r in records]) for s in range(K)]).astype(np.int32)
    ncol = np.array([[r['ncol'][s] for r in records] for s in range(K)], np.int32).reshape(-1)
    cat = lambda xs, dt: np.ascontiguousarray(np.concatenate(xs) if xs else np.zeros(0), dtype=dt)
    return {'W': W, 'K': K, 'first_body': first_body, 'bodies': np.ascontiguousarray(bodies, np.float64), 'step_man': step_man, 'step_pt': step_pt,
            'man_bodies': cat(mb, np.int32), 'basis': cat(basis, np.float64), 'anchors': cat(anchors, np.float64), 'pt_man': cat(pt_man, np.int32),
            'pt_prev': cat(pt_prev, np.int32), 'colors': colors, 'ncol': ncol, 'params': records[0]['params'], 'nb': int(first_body[-1])}


def split(c: dict, w: int, params: dict) -> dict:
    """World w of a combined recording as one world's recording (indices over its own steps): the
    inverse of `combine` for one world."""
    W, K = c['W'], c['K']
    fb = c.get('first_body')
    sm, sp = c['step_man'].reshape(K, W + 1), c['step_pt'].reshape(K, W + 1)
    bodies_of = lambda arr, per: arr.reshape(K, -1)[:, b0 * per:b1 * per].reshape(-1)
    if fb is None:
        raise ValueError('the recording needs first_body')
    b0, b1 = int(fb[w]), int(fb[w + 1])
    n = b1 - b0
    mb, basis, anchors, pt_man, pt_prev = [], [], [], [], []
    step_man, step_pt = np.zeros(K + 1, np.int32), np.zeros(K + 1, np.int32)
    m = p = 0
    for s in range(K):
        m0, m1, p0, p1 = int(sm[s, w]), int(sm[s, w + 1]), int(sp[s, w]), int(sp[s, w + 1])
        step_man[s], step_pt[s] = m, p
        mb.append(c['man_bodies'][2 * m0:2 * m1])
        basis.append(c['basis'][9 * m0:9 * m1])
        anchors.append(c['anchors'][6 * p0:6 * p1])
        pt_man.append(c['pt_man'][p0:p1] - m0 + m)
        prev = c['pt_prev'][p0:p1]
        if s > 0:
            prev = np.where(prev >= 0, prev - int(sp[s - 1, w]) + int(step_pt[s - 1]), -1)
        pt_prev.append(prev)
        m += m1 - m0
        p += p1 - p0
    step_man[K], step_pt[K] = m, p
    cat = lambda xs, dt: np.ascontiguousarray(np.concatenate(xs) if xs else np.zeros(0), dtype=dt)
    return {'n': n, 'steps': K, 'bodies': c['bodies'][13 * b0:13 * b1].copy(), 'step_man': step_man, 'step_pt': step_pt,
            'man_bodies': cat(mb, np.int32), 'basis': cat(basis, np.float64), 'anchors': cat(anchors, np.float64),
            'pt_man': cat(pt_man, np.int32), 'pt_prev': cat(pt_prev, np.int32),
            'colors': bodies_of(c['colors'], 1).astype(np.int32), 'ncol': c['ncol'].reshape(K, W)[:, w].astype(np.int32).copy(),
            'params': params, 'manifolds': m, 'points': p}


class Adjoint:
    """Double-precision replay and reverse sweep on one B200 for a batch of recorded worlds."""

    def __init__(self, records: list, checkpoint: int = 10, device: int = 0):
        self.lib = _abi.load()
        c = combine(records)
        self._keep = c
        P = c['params']
        ptr = lambda a: a.ctypes.data if a.size else None
        d = AdjointDesc(worlds=c['W'], steps=c['K'], iterations=int(P['iterations']), checkpoint=checkpoint, dt=P['dt'], gravity=P['gravity'],
                        alpha=P['alpha'], gamma=P['gamma'], beta_lin=P['beta_lin'], contact_margin=P['contact_margin'],
                        world_first_body=ptr(c['first_body']), bodies=ptr(c['bodies']), step_first_manifold=ptr(c['step_man']),
                        step_first_point=ptr(c['step_pt']), manifold_bodies=ptr(c['man_bodies']), manifold_basis=ptr(c['basis']),
                        point_anchors=ptr(c['anchors']), point_manifold=ptr(c['pt_man']), point_prev=ptr(c['pt_prev']), colors=ptr(c['colors']),
                        color_counts=ptr(c['ncol']), device=device)
        self.handle = ctypes.c_void_p()
        code = self.lib.avbd_adjoint_create(ctypes.byref(d), ctypes.byref(self.handle))
        if code != _abi.AVBD_OK:
            raise _abi.error(code, 'avbd_adjoint_create failed')
        self.worlds, self.bodies = c['W'], c['nb']
        self.first_body = c['first_body']

    @classmethod
    def from_batch(cls, batch, checkpoint: int = 10) -> 'Adjoint':
        """The adjoint of a batch's finished recording (BatchSolver3D.record_start): the device
        recording is adopted as is; the batch keeps its worlds but no longer the recording."""
        self = cls.__new__(cls)
        self.lib = _abi.load()
        self._keep = None
        self.handle = ctypes.c_void_p()
        code = self.lib.avbd_adjoint_create_from_batch(batch.handle, checkpoint, ctypes.byref(self.handle))
        if code != _abi.AVBD_OK:
            msg = self.lib.avbd_batch_last_error(batch.handle)
            raise _abi.error(code, 'avbd_adjoint_create_from_batch: ' + (msg.decode() if msg else ''))
        info = self.info()
        self.worlds, self.bodies = info['worlds'], info['bodies']
        self.first_body = np.array([batch.world_info(w)['first_body'] for w in range(self.worlds)] + [self.bodies], np.uint32)
        return self

    def info(self) -> dict:
        u = [ctypes.c_uint32() for _ in range(4)]
        q = [ctypes.c_uint64() for _ in range(2)]
        self._check(self.lib.avbd_adjoint_info(self.handle, *[ctypes.byref(x) for x in u + q]))
        return dict(zip(('worlds', 'steps', 'bodies', 'max_points', 'manifolds', 'points'), [x.value for x in u + q]))

    def read_recording(self) -> dict:
        """The recording in the layout `combine` builds (all worlds, global indices)."""
        info = self.info()
        W, K, nb, nm, npts = info['worlds'], info['steps'], info['bodies'], info['manifolds'], info['points']
        c = {'W': W, 'K': K, 'nb': nb, 'bodies': np.zeros(13 * nb), 'step_man': np.zeros(K * (W + 1), np.int32),
             'step_pt': np.zeros(K * (W + 1), np.int32), 'man_bodies': np.zeros(2 * max(nm, 1), np.int32), 'basis': np.zeros(9 * max(nm, 1)),
             'anchors': np.zeros(6 * max(npts, 1)), 'pt_man': np.zeros(max(npts, 1), np.int32), 'pt_prev': np.zeros(max(npts, 1), np.int32),
             'colors': np.zeros(K * nb, np.int32), 'ncol': np.zeros(K * W, np.int32)}
        keys = ('bodies', 'step_man', 'step_pt', 'man_bodies', 'basis', 'anchors', 'pt_man', 'pt_prev', 'colors', 'ncol')
        self._check(self.lib.avbd_adjoint_read_recording(self.handle, *[c[k].ctypes.data for k in keys]))
        c['first_body'] = self.first_body
        return c

    def nominal(self) -> np.ndarray:
        """The parameters the recorded rollout ran with (8 per body: v0, omega0, mass, friction)."""
        p = np.zeros(8 * self.bodies)
        self._check(self.lib.avbd_adjoint_nominal(self.handle, p.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return p

    def destroy(self):
        if getattr(self, 'handle', None) and self.handle.value:
            self.lib.avbd_adjoint_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _check(self, code):
        if code != _abi.AVBD_OK:
            msg = self.lib.avbd_adjoint_last_error(self.handle)
            raise _abi.error(code, msg.decode() if msg else '')

    def set_target(self, target: np.ndarray):
        t = np.ascontiguousarray(target, np.float64).reshape(-1)
        self._check(self.lib.avbd_adjoint_set_target(self.handle, t.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def forward(self, params: np.ndarray):
        """Loss per world and final poses (7 per body)."""
        p = np.ascontiguousarray(params, np.float64).reshape(-1)
        loss = np.zeros(self.worlds)
        fin = np.zeros(7 * self.bodies)
        D = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.avbd_adjoint_forward(self.handle, p.ctypes.data_as(D), loss.ctypes.data_as(D), fin.ctypes.data_as(D)))
        return loss, fin.reshape(-1, 7)

    def backward(self, params: np.ndarray):
        """Loss per world and the gradient (8 per body: v0, omega0, mass, friction)."""
        p = np.ascontiguousarray(params, np.float64).reshape(-1)
        loss = np.zeros(self.worlds)
        g = np.zeros(8 * self.bodies)
        D = ctypes.POINTER(ctypes.c_double)
        self._check(self.lib.avbd_adjoint_backward(self.handle, p.ctypes.data_as(D), g.ctypes.data_as(D), loss.ctypes.data_as(D)))
        return loss, g
