"""The host hull builder (avbd_hull_build, a restatement of src/avbd3d/hull.ts convexHull) against
the reference's own hull tests (tests/hull.test.ts:15-130), through the C ABI. Host code: no GPU."""

import math

import numpy as np

from avbd_b200.hulls import build_hull


def close(a, b, eps=1e-5):
    assert abs(a - b) <= eps, f'{a} vs {b}'


def box(w, h, d):
    out = []
    for x in (-w / 2, w / 2):
        for y in (-h / 2, h / 2):
            for z in (-d / 2, d / 2):
                out += [x, y, z]
    return out


def park_miller(seed):
    s = [seed]

    def rnd():
        s[0] = (s[0] * 16807) % 2147483647
        return s[0] / 2147483647
    return rnd


def euler(h):
    return len(h.vertices) - len(h.edges) + len(h.faces)


def test_box_faces_edges_volume_moments(cuda_lib):
    """hull.test.ts:15-28: six quad faces, twelve edges, its volume and moments (inner points dropped)."""
    h = build_hull(box(2, 1, 0.5) + [0, 0, 0, 0.3, 0.1, 0.1])
    assert len(h.faces) == 6 and all(len(f[2]) == 4 for f in h.faces)
    assert len(h.edges) == 12 and len(h.vertices) == 8
    close(h.volume, 1)
    m = sorted(h.moments)
    close(m[0], (1 + 0.25) / 12, 1e-6)
    close(m[1], (4 + 0.25) / 12, 1e-6)
    close(m[2], (4 + 1) / 12, 1e-6)
    close(h.radius, math.hypot(1, 0.5, 0.25))


def test_faces_are_planes_and_edges_join_two_faces(cuda_lib):
    """hull.test.ts:30-47: every vertex behind every face, V - E + F = 2, each edge on its two faces."""
    r = park_miller(7)
    pts = []
    for _ in range(200):
        pts += [(r() * 2 - 1) * 1.5 + 3, (r() * 2 - 1) * 0.7 - 2, r() * 2 - 1]
    h = build_hull(pts)
    v = h.vertices
    for n, d, _ in h.faces:
        close(float(np.linalg.norm(n)), 1)
        assert np.all(v @ n <= d + 1e-5)
    assert euler(h) == 2
    faces = h.faces
    for a, b, f, g in h.edges:
        assert a in faces[f][2] and b in faces[f][2] and a in faces[g][2] and b in faces[g][2]


def test_principal_frame_maps_back_onto_the_points(cuda_lib):
    """hull.test.ts:49-72: a turned and moved box; centre, sizes, and every vertex back on a corner."""
    ang = math.pi / 6
    c, s = math.cos(ang), math.sin(ang)
    src = box(3, 1, 0.4)
    turned = []
    for i in range(0, len(src), 3):
        turned += [c * src[i] - s * src[i + 1] + 1, s * src[i] + c * src[i + 1] - 2, src[i + 2] + 0.5]
    h = build_hull(turned)
    assert [round(x * 1e6) / 1e6 for x in h.center] == [1, -2, 0.5]
    sizes = sorted(h.size)
    close(sizes[0], 0.4)
    close(sizes[1], 1)
    close(sizes[2], 3)
    x, y, z, w = h.rotation
    T = np.array(turned).reshape(-1, 3)
    for p in h.vertices:
        t = [2 * (y * p[2] - z * p[1]), 2 * (z * p[0] - x * p[2]), 2 * (x * p[1] - y * p[0])]
        q = np.array([p[0] + w * t[0] + (y * t[2] - z * t[1]), p[1] + w * t[1] + (z * t[0] - x * t[2]),
                      p[2] + w * t[2] + (x * t[1] - y * t[0])]) + np.array(h.center)
        assert np.min(np.linalg.norm(T - q, axis=1)) < 1e-5


def test_flat_and_tiny_point_sets_have_no_hull(cuda_lib):
    """hull.test.ts:74-77."""
    assert build_hull([0, 0, 0, 1, 0, 0, 0, 1, 0]) is None
    assert build_hull([0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1, 0, 0.5, 0.5, 0]) is None


def test_fracture_piece_points_on_planes(cuda_lib):
    """hull.test.ts:79-102: a cube corner cut by a slanted plane, many points on every face."""
    r = park_miller(11)
    pts = []
    for k in range(400):
        face = k % 4
        u, v = r(), r()
        p = [0, u, v] if face == 0 else [u, 0, v] if face == 1 else [u, v, 0] if face == 2 else [u, v, 1.6 - u - v]
        ok = (0 <= p[2] <= 1) if face == 3 else (p[0] + p[1] + p[2] <= 1.6)
        if ok:
            pts += p
    for c in ([0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0.6, 0], [0.6, 1, 0], [1, 0, 0.6], [0, 1, 0.6], [0.6, 0, 1], [0, 0.6, 1]):
        pts += c
    h = build_hull(pts)
    assert euler(h) == 2
    assert len(h.faces) == 7
    faces = h.faces
    for a, b, f, g in h.edges:
        assert f != g and a in faces[f][2] and b in faces[g][2]
    close(h.volume, 1 - (1.4 ** 3 - 3 * 0.4 ** 3) / 6, 1e-4)


def test_sphere_points_simplified_to_the_vertex_limit(cuda_lib):
    """hull.test.ts:104-121: points on a sphere, simplified to at most 32 vertices by farthest-point sampling."""
    r = park_miller(3)
    last = 0.0
    for n in (100, 400):
        pts = []
        for _ in range(n):
            u = r() * 2 - 1
            a = r() * 2 * math.pi
            rr = math.sqrt(1 - u * u)
            pts += [rr * math.cos(a), rr * math.sin(a), u]
        h = build_hull(pts)
        assert len(h.vertices) == min(n, 32)
        assert len(h.faces) <= 255 and len(h.edges) <= 255
        assert euler(h) == 2
        assert max(last * 0.95, 3) < h.volume < 4 / 3 * math.pi
        last = h.volume
