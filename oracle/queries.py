"""CPU restatement of the passes a World runs around the step (TEST INFRASTRUCTURE: imported only by
tests/, never by the product), in double precision from the same f32 records the device holds:

  pushes          src/lib/push.ts:23-37 (the shader) and :50-58 (addImpulse)
  contact events  src/lib/contacts.ts:93-125 (touching, ended), as sets of lifetime-ID pairs
  raycasts        src/lib/raycast.ts:80-150 (trace), :16-45 (nearest hit, lowest body on ties)
"""

from __future__ import annotations

import numpy as np


def rotate(q, v):
    """The reference's rotate (ref/math.ts:115-126): t = 2 u x v; v + t w + u x t."""
    u, w = np.asarray(q[:3], float), float(q[3])
    t = 2.0 * np.cross(u, v)
    return np.asarray(v, float) + t * w + np.cross(u, t)


def conj(q):
    return np.array([-q[0], -q[1], -q[2], q[3]], float)


def apply_pushes(bodies: np.ndarray, pushes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Velocities and angular velocities after the pushes (push.ts:23-37): a dynamic enabled body gains
    lin / m and, in its principal frame, (moment - x cross off_lin) / I."""
    vel = bodies['vel'].astype(float).copy()
    avel = bodies['ang_vel'].astype(float).copy()
    for p in pushes:
        b = int(p['body'])
        if (int(bodies['flags'][b]) & 2) or bodies['mass'][b] <= 0:
            continue
        m = float(bodies['mass'][b])
        vel[b] += p['lin'].astype(float) / m
        q = bodies['rot'][b].astype(float)
        L = p['moment'].astype(float) - np.cross(bodies['pos'][b].astype(float), p['off_lin'].astype(float))
        local = rotate(conj(q), L) / np.maximum(bodies['moment'][b].astype(float), 1e-12)
        avel[b] += rotate(q, local)
    return vel, avel


def touching_pairs(manifolds: np.ndarray, watch: dict) -> dict:
    """This step's set (contacts.ts:93-103): lifetime-ID pairs of the touching pairs that have a
    reporting body; watch maps slot -> (id, reporting)."""
    out = {}
    for i, m in enumerate(manifolds):
        a, b = int(m['a']), int(m['b'])
        if m['count'] == 0 or a not in watch or b not in watch:
            continue
        (ia, ra), (ib, rb) = watch[a], watch[b]
        if ia and ib and (ra or rb):
            out[(ia, ib)] = i
    return out


def contact_events(prev: set, manifolds: np.ndarray, contacts: np.ndarray, bodies: np.ndarray, watch: dict, step: int, dt: float):
    """This step's begin events (where, how hard, the normal: contacts.ts:104-114) and end events
    (:117-125), and this step's set."""
    now = touching_pairs(manifolds, watch)
    events = []
    for key, i in now.items():
        if key in prev:
            continue
        m = manifolds[i]
        a = int(m['a'])
        pts = contacts[int(m['first']):int(m['first']) + int(m['count'])]
        pA, qA = bodies['pos'][a].astype(float), bodies['rot'][a].astype(float)
        point = np.mean([rotate(qA, c['r_a'].astype(float)) + pA for c in pts], axis=0)
        impulse = abs(float(np.sum(pts['lam'][:, 0].astype(float)))) * dt
        events.append((1, key[0], key[1], step, point, impulse, m['normal'].astype(float)))
    for key in prev:
        if key not in now:
            events.append((2, key[0], key[1], step, np.zeros(3), 0.0, np.zeros(3)))
    return events, set(now)


def _planes(body, hull_words):
    """A box's or hull's face planes in its frame: (normal, offset) rows."""
    shape = float(body['shape'])
    size = body['size'].astype(float)
    if shape > 2.5:
        head = hull_words[4 * int(shape - 3 + 0.5):4 * int(shape - 3 + 0.5) + 4]
        fs, faces = int(head[2]), int(head[3])
        return [hull_words[4 * (fs + 2 * k):4 * (fs + 2 * k) + 4].view(np.float32).astype(float) for k in range(faces)]
    planes = []
    for k in range(6):
        e = np.zeros(3)
        e[k // 2] = 1.0 if k % 2 == 0 else -1.0
        planes.append(np.array([e[0], e[1], e[2], size[k // 2] * 0.5]))
    return planes


def normals_at(body, hull_words, origin, direction, t, tol):
    """The world normals a hit at ray parameter t may report: a sphere's at the point o + d t (a
    grazing ray's normal moves by the distance's rounding over the radius, so it is taken at the
    distance the device found), a box's or hull's faces that the ray enters within `tol` of t (the
    faces that tie where it lands on an edge or a corner)."""
    q = body['rot'].astype(float)
    o = rotate(conj(q), np.asarray(origin, float) - body['pos'].astype(float))
    d = rotate(conj(q), np.asarray(direction, float))
    if abs(float(body['shape']) - 1.0) < 0.5:
        p = o + d * t
        wn = rotate(q, p / np.linalg.norm(p))
        return [wn / np.linalg.norm(wn)]
    out = []
    for pl in _planes(body, hull_words):
        denom = pl[:3] @ d
        if denom < -1e-12 and abs((pl[3] - pl[:3] @ o) / denom - t) <= tol:
            wn = rotate(q, pl[:3])
            out.append(wn / np.linalg.norm(wn))
    return out


def ray_trace(body, hull_words, origin, direction, max_distance):
    """Ray against one body (raycast.ts:80-150): (distance, normal in the body's frame) or None."""
    q = body['rot'].astype(float)
    size = body['size'].astype(float)
    shape = float(body['shape'])
    o = rotate(conj(q), np.asarray(origin, float) - body['pos'].astype(float))
    d = rotate(conj(q), np.asarray(direction, float))
    if abs(shape - 1.0) < 0.5:
        radius = size[0] * 0.5
        bh = o @ d
        c = o @ o - radius * radius
        disc = bh * bh - c
        if disc < 0:
            return None
        t = -bh - np.sqrt(disc)
        if c <= 0:
            t, n = 0.0, -d
        else:
            if t < 0:
                return None
            p = o + d * t
            n = p / np.linalg.norm(p)
    else:
        tin, tout, n = -3.0e38, 3.0e38, np.zeros(3)
        for pl in _planes(body, hull_words):
            denom = pl[:3] @ d
            dist = pl[3] - pl[:3] @ o
            if abs(denom) < 1e-12:
                if dist < 0:
                    return None
                continue
            s = dist / denom
            if denom < 0:
                if s > tin:
                    tin, n = s, pl[:3]
            else:
                tout = min(tout, s)
            if tin > tout:
                return None
        if tout < 0:
            return None
        t = tin
        if t <= 0:
            t, n = 0.0, -d
    if t > max_distance:
        return None
    return max(t, 0.0), n


def raycast(bodies: np.ndarray, hull_words, filters: np.ndarray, origin, direction, max_distance=3.0e38, ignore=(), mask=0xFFFFFFFF):
    """The nearest hit among the bodies (the lowest slot on ties): (body, distance, world normal) or None."""
    d = np.asarray(direction, float)
    l = np.linalg.norm(d)
    d = d / l if l > 0 else d
    best = None
    for b in range(len(bodies)):
        if (int(bodies['flags'][b]) & 2) or b in ignore or (int(filters[b][0]) & mask) == 0:
            continue
        h = ray_trace(bodies[b], hull_words, origin, d, max_distance)
        if h is not None and (best is None or h[0] < best[1]):
            best = (b, h[0], h[1])
    if best is None:
        return None
    b, t, n = best
    wn = rotate(bodies['rot'][b].astype(float), n)
    return b, t, wn / np.linalg.norm(wn)
