"""The host hull builder (avbd_hull_build) on degenerate point sets, by the reference's own procedure
(tests/hull-degenerate.test.ts): a Voronoi glass fragment (the reference's fixture, copied by
tests/golden/copy_hull_fixture.py), 400 seeded fracture-like clouds (points on faces and edges,
inside, near-coincident corner clusters, duplicates, 1 µm to 10 m, plates) and 120 flat, linear or
clustered sets. Each must finish fast and give a closed convex hull holding its points (or, for
the flat sets, no hull). Host code: no GPU."""

import json
import math
import os
import time

import numpy as np

from avbd_b200.hulls import build_hull

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
MAX_HULL_VERTICES = 32


def _random(seed):
    """hull-degenerate.test.ts:113-117: seeded uniform [0, 1) (Park-Miller)."""
    s = [seed]

    def rnd():
        s[0] = (s[0] * 16807) % 2147483647
        return s[0] / 2147483647
    return rnd


def _rot(q, v):
    x, y, z, w = q
    t = np.array([2 * (y * v[2] - z * v[1]), 2 * (z * v[0] - x * v[2]), 2 * (x * v[1] - y * v[0])])
    return np.array([v[0] + w * t[0] + (y * t[2] - z * t[1]), v[1] + w * t[1] + (z * t[0] - x * t[2]), v[2] + w * t[2] + (x * t[1] - y * t[0])])


def _to_input(h, v):
    """A principal-frame point in the input frame (:36-41)."""
    return _rot(h.rotation, v) + np.asarray(h.center)


def _to_local(h, pts):
    """Input points into the principal frame: Rᵀ(p - centre) (:27-33)."""
    x, y, z, w = h.rotation
    conj = (-x, -y, -z, w)
    return np.array([_rot(conj, p - np.asarray(h.center)) for p in pts])


def _scale(points):
    p = np.asarray(points, np.float64).reshape(-1, 3)
    e = p.max(axis=0) - p.min(axis=0)
    return float(e.max()), float(np.abs(p).max()), float(np.prod(e))


def _assert_convex(h, eps, label):
    """:59-75: a closed convex polyhedron."""
    n = len(h.vertices)
    assert 4 <= n <= MAX_HULL_VERTICES, f'{label}: {n} vertices'
    assert len(h.faces) <= 255 and len(h.edges) <= 255, label
    assert n - len(h.edges) + len(h.faces) == 2, f'{label}: Euler'
    v = h.vertices
    for normal, d, idx in h.faces:
        assert abs(np.linalg.norm(normal) - 1) < 1e-6, label
        s = v @ normal - d
        assert s.max() <= eps, f'{label}: a vertex {s.max()} in front of a face'
        assert s[idx].min() >= -eps, f'{label}: face not planar ({s[idx].min()})'
    for a, b, f, g in h.edges.tolist():
        assert f != g and a in h.faces[f][2] and b in h.faces[g][2], label
    assert h.volume > 0 and all(m > 0 for m in h.moments), label


def _outside(h, points):
    """:78-88: most any input point is in front of any face."""
    loc = _to_local(h, np.asarray(points, np.float64).reshape(-1, 3))
    worst = -math.inf
    for normal, d, _ in h.faces:
        worst = max(worst, float((loc @ normal - d).max()))
    return worst


def _timed(points):
    t0 = time.perf_counter()
    h = build_hull(points)
    return h, (time.perf_counter() - t0) * 1000


def test_glass_fragment(cuda_lib):
    """:90-105: 238 points of a 4.8 x 3.8 x 3.9 cm fragment: a hull, fast, holding every point."""
    points = np.array(json.load(open(os.path.join(GOLDEN, 'hull-fracture-glass.json'))), np.float32)
    assert len(points) == 238 * 3
    h, ms = _timed(points)
    assert h is not None and ms < 500, ms
    extent, _, box = _scale(points)
    _assert_convex(h, 1e-6 * extent, 'fragment')
    assert len(h.vertices) < MAX_HULL_VERTICES
    assert _outside(h, points) <= 1e-6 * extent
    assert 0.3 * box < h.volume < box
    assert all(s <= 2 * extent for s in h.size)


def _fracture_cloud(rnd):
    """:119-168: a fracture-like piece, its clean hull and how far its clusters reach."""
    scale = 10 ** (rnd() * 7 - 6)
    axes = [scale * (0.2 + 0.8 * rnd()), scale * (0.2 + 0.8 * rnd()), scale * (0.2 + 0.8 * rnd())]
    if rnd() < 0.25:
        k = math.floor(rnd() * 3)
        axes[k] *= 10 ** (-1 - 2 * rnd())
    offset = [(rnd() - 0.5) * 8 * scale for _ in range(3)]
    corners = []
    for _ in range(4 + math.floor(rnd() * 9)):
        for k in range(3):
            corners.append(offset[k] + (rnd() - 0.5) * axes[k])
    clean = build_hull(np.array(corners, np.float32))
    verts = [_to_input(clean, v) for v in clean.vertices]

    def mix(ws, vs):
        t = sum(ws)
        return sum((w / t) * np.asarray(v) for w, v in zip(ws, vs))
    out = list(verts)
    for _ in range(20 + math.floor(rnd() * 150)):
        f = clean.faces[math.floor(rnd() * len(clean.faces))]
        out.append(mix([rnd() ** 3 for _ in f[2]], [verts[v] for v in f[2]]))
    for _ in range(math.floor(rnd() * 40)):
        a, b = clean.edges[math.floor(rnd() * len(clean.edges))][:2]
        t = rnd()
        out.append(mix([t, 1 - t], [verts[a], verts[b]]))
    for _ in range(math.floor(rnd() * 30)):
        out.append(mix([rnd() ** 4 for _ in verts], verts))
    reach = 0.0
    for _ in range(math.floor(rnd() * 4)):
        v = verts[math.floor(rnd() * len(verts))]
        for _ in range(1 + math.floor(rnd() * 3)):
            r = 10 ** (-9 + 5 * rnd()) * scale
            reach = max(reach, r)
            out.append(np.array([v[0] + (rnd() - 0.5) * r, v[1] + (rnd() - 0.5) * r, v[2] + (rnd() - 0.5) * r]))
    for _ in range(math.floor(rnd() * 30)):
        out.append(np.array(out[math.floor(rnd() * len(out))]))
    for i in range(len(out) - 1, 0, -1):
        j = math.floor(rnd() * (i + 1))
        out[i], out[j] = out[j], out[i]
    return np.array(out, np.float64).astype(np.float32).reshape(-1), clean, reach


def _surface_area(h):
    area = 0.0
    v = h.vertices
    for _, _, idx in h.faces:
        for j in range(1, len(idx) - 1):
            area += np.linalg.norm(np.cross(v[idx[j]] - v[idx[0]], v[idx[j + 1]] - v[idx[0]])) / 2
    return area


def test_fracture_like_sets(cuda_lib):
    """:170-207: 400 seeded clouds finish, convex and containing their points."""
    rnd = _random(20261102)
    contained = 0
    for k in range(400):
        points, clean, reach = _fracture_cloud(rnd)
        h, ms = _timed(points)
        label = f'case {k}'
        assert ms < 1000, f'{label}: {ms} ms'
        assert h is not None, f'{label}: no hull'
        extent, magnitude, box = _scale(points)
        tol = 2e-5 * max(extent, magnitude)
        _assert_convex(h, tol, label)
        if len(h.vertices) < MAX_HULL_VERTICES:
            contained += 1
            s = _outside(h, points)
            assert s <= tol, f'{label}: a point {s} outside (size {extent})'
        assert h.volume <= box * (1 + 1e-3), label
        assert h.volume >= clean.volume * 0.98, f'{label}: volume {h.volume} vs {clean.volume}'
        assert h.volume <= clean.volume * 1.02 + _surface_area(clean) * (reach + tol), label
    assert contained > 0.9 * 400, contained


def test_flat_linear_and_clustered_sets(cuda_lib):
    """:209-233: sets flat or in one place to within rounding finish: no hull, or a valid one."""
    rnd = _random(77)
    for k in range(120):
        scale = 10 ** (rnd() * 6 - 5)
        out = []
        kind = k % 3
        for _ in range(50 + math.floor(rnd() * 200)):
            u, v = rnd() - 0.5, rnd() - 0.5
            off = (rnd() - 0.5) * 1e-8
            if kind == 0:
                p = [u, v, 0.3 * u - 0.7 * v + off]
            elif kind == 1:
                p = [u, 0.5 * u + off, -u + off]
            else:
                p = [off, off * rnd(), off * rnd()]
            out += [x * scale + 0.25 * scale for x in p]
            if rnd() < 0.2:
                out += out[-3:]
        pts = np.array(out, np.float64).astype(np.float32)
        h, ms = _timed(pts)
        assert ms < 1000, f'set {k}: {ms} ms'
        if h is not None:
            extent, magnitude, _ = _scale(pts)
            tol = 2e-5 * max(extent, magnitude)
            _assert_convex(h, tol, f'set {k}')
            assert _outside(h, pts) <= tol, f'set {k}'
