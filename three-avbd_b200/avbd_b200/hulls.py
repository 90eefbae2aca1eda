"""Convex hull shapes (src/avbd3d/hull.ts, shapes.ts hull()) through the C ABI's host builder.

`build_hull(points)` is the reference's `convexHull(points)`: the hull record in the reference's
packed layout (gpu/solver.ts:313-338, header at vec4 0) and the mass properties. The builder is
host code in the CUDA library and needs no device.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _abi


@dataclass
class HullShape:
    packed: np.ndarray  # uint32, 4 words per vec4, header at vec4 0
    volume: float
    moments: tuple
    size: tuple
    radius: float
    center: tuple
    rotation: tuple

    @property
    def vec4s(self) -> int:
        return len(self.packed) // 4

    def header(self):
        return [int(x) for x in self.packed[:8]]

    @property
    def vertices(self) -> np.ndarray:
        vs, nv = self.header()[:2]
        return self.packed[4 * vs:4 * (vs + nv)].view(np.float32).reshape(-1, 4)[:, :3].astype(np.float64)

    @property
    def faces(self) -> list:
        """(normal, d, vertex indices) per face."""
        vs, nv, fs, nf, es, ne, is_, _ = self.header()
        out = []
        for k in range(nf):
            rec = self.packed[4 * (fs + 2 * k):4 * (fs + 2 * k) + 8]
            plane = rec[:4].view(np.float32).astype(np.float64)
            first, count = int(rec[4]), int(rec[5])
            idx = [int(self.packed[4 * is_ + first + j]) for j in range(count)]
            out.append((plane[:3], float(plane[3]), idx))
        return out

    @property
    def edges(self) -> np.ndarray:
        vs, nv, fs, nf, es, ne, is_, _ = self.header()
        return self.packed[4 * es:4 * (es + ne)].reshape(-1, 4).astype(np.int64)


def build_hull(points) -> HullShape | None:
    """convexHull(points) (hull.ts:60-75): None when the points span no volume."""
    lib = _abi.load()
    pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1)
    n = len(pts) // 3
    size = ctypes.c_uint32()
    props = _abi.HullProps()
    code = lib.avbd_hull_build(pts.ctypes.data_as(ctypes.c_void_p), n, None, 0, ctypes.byref(size), ctypes.byref(props))
    if code == _abi.AVBD_ERR_INVALID:
        return None
    if code != _abi.AVBD_OK:
        raise _abi.AvbdError(code, 'avbd_hull_build failed')
    packed = np.zeros(4 * size.value, dtype=np.uint32)
    code = lib.avbd_hull_build(pts.ctypes.data_as(ctypes.c_void_p), n, _abi.uptr(packed), size.value, ctypes.byref(size), ctypes.byref(props))
    if code != _abi.AVBD_OK:
        raise _abi.AvbdError(code, 'avbd_hull_build failed')
    return HullShape(packed, props.volume, tuple(props.moments), tuple(props.size), props.radius, tuple(props.center), tuple(props.rotation))


def relocate(packed: np.ndarray, at: int) -> np.ndarray:
    """A record with its header at vec4 `at` of a hull buffer (packHull(shape, at))."""
    out = packed.copy()
    for k in (0, 2, 4, 6):
        out[k] += at
    return out
