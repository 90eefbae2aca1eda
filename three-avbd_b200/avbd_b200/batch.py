"""Batched worlds over the C ABI (avbd_batch_* in include/avbd.h).

The reference steps one world per GpuSolver3D and has no batched mode. `BatchSolver3D` holds many
small independent worlds (up to 4096 bodies each) on one B200 and steps them all with two launches
per step; each world runs exactly the single-world step on its own bodies, with its own indices.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import BODY_DTYPE, INFO_DTYPE, JOINT_DTYPE, BatchConfig, BatchStatus, BatchTuning, BatchWorld, Counters, ptr, uptr
from .scenes import Scene
from .solver import CudaSolver3D, scene_records, to_params


class BatchSolver3D:
    """Independent worlds sharing one parameter set. Worlds come from scenes (`add_scene`), from host
    records (`add_world`) or from a single world whose state they continue (`add_world_from`)."""

    def __init__(self, world_capacity: int, body_capacity: int, joint_capacity: int = 0, *, params=None, pairs_per_body: int = 0,
                 device: int = 0):
        self.lib = _abi.load()
        cfg = BatchConfig(world_capacity=world_capacity, body_capacity=body_capacity, joint_capacity=max(joint_capacity, 1),
                          pairs_per_body=pairs_per_body, device=device)
        self.handle = ctypes.c_void_p()
        code = self.lib.avbd_batch_create(ctypes.byref(cfg), ctypes.byref(self.handle))
        if code != _abi.AVBD_OK:
            raise _abi.error(code, 'avbd_batch_create failed (a B200 with the CUDA library is required; there is no CPU fallback)')
        if params is not None:
            self.set_params(params)

    def destroy(self):
        if getattr(self, 'handle', None) and self.handle.value:
            self.lib.avbd_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _check(self, code: int):
        if code != _abi.AVBD_OK:
            msg = self.lib.avbd_batch_last_error(self.handle)
            raise _abi.error(code, msg.decode() if msg else '')

    def set_params(self, sp):
        self._check(self.lib.avbd_batch_set_params(self.handle, ctypes.byref(to_params(sp))))

    # --- worlds ---
    def add_world(self, bodies: np.ndarray, joints: np.ndarray | None = None, infos: np.ndarray | None = None,
                  ignores: np.ndarray | None = None) -> int:
        bodies = np.ascontiguousarray(bodies, dtype=BODY_DTYPE)
        joints = np.ascontiguousarray(joints if joints is not None else np.zeros(0, JOINT_DTYPE), dtype=JOINT_DTYPE)
        infos = np.ascontiguousarray(infos if infos is not None else np.zeros(0, INFO_DTYPE), dtype=INFO_DTYPE)
        ignores = np.ascontiguousarray(ignores if ignores is not None else np.zeros((0, 2), np.uint32), dtype=np.uint32).reshape(-1, 2)
        index = ctypes.c_uint32()
        self._check(self.lib.avbd_batch_add_world(self.handle, ptr(bodies), len(bodies), ptr(joints) if len(joints) else None,
                                                  ptr(infos) if len(infos) else None, len(joints), uptr(ignores) if len(ignores) else None,
                                                  len(ignores), ctypes.byref(index)))
        return index.value

    def add_scene(self, scene: Scene) -> int:
        bodies, joints, infos, ignores = scene_records(scene)
        return self.add_world(bodies, joints, infos, ignores)

    def add_world_from(self, world: CudaSolver3D) -> int:
        index = ctypes.c_uint32()
        self._check(self.lib.avbd_batch_add_world_from(self.handle, world.handle, ctypes.byref(index)))
        return index.value

    def world_info(self, w: int) -> dict:
        out = BatchWorld()
        self._check(self.lib.avbd_batch_world_info(self.handle, w, ctypes.byref(out)))
        return {n: getattr(out, n) for n, _ in out._fields_}

    def info(self) -> dict:
        out = BatchStatus()
        self._check(self.lib.avbd_batch_info(self.handle, ctypes.byref(out)))
        return {n: getattr(out, n) for n, _ in out._fields_}

    @property
    def world_count(self) -> int:
        return self.info()['worlds']

    # --- stepping ---
    def step(self, n: int = 1):
        self._check(self.lib.avbd_batch_step(self.handle, n))

    def synchronize(self):
        self._check(self.lib.avbd_batch_synchronize(self.handle))

    def use_graphs(self, on: bool = True):
        self._check(self.lib.avbd_batch_use_graphs(self.handle, 1 if on else 0))

    def tune(self, steps: int = 3) -> dict:
        """Times every candidate launch shape over `steps` real steps each and keeps the fastest."""
        t = BatchTuning()
        self._check(self.lib.avbd_batch_tune(self.handle, steps, ctypes.byref(t)))
        k = t.candidates
        return {'candidates': [{'collide_threads': t.candidate_threads[i], 'solve_blocks': t.candidate_solve_blocks[i],
                                'rows_per_lane': t.candidate_rows_per_lane[i], 'world_threads': t.candidate_world_threads[i],
                                'ms_per_step': t.candidate_ms[i]} for i in range(k)],
                'collide_threads': t.collide_threads, 'solve_blocks': t.solve_blocks, 'rows_per_lane': t.rows_per_lane,
                'world_threads': t.world_threads, 'ms_per_step': t.ms_per_step, 'steps_taken': t.steps_taken}

    def set_launch(self, collide_threads: int = 128, solve_blocks: int = 0, rows_per_lane: int = 1, world_threads: int = 256):
        """Sets the launch shape the tuner would pick: collision block size (64, 128, 256), solve blocks (0:
        as many as fit), the least rows a lane (1..8), and the solve's threads a world (256: a block a
        world; 128, 64 or 32: two, four or eight worlds a block). Results are the same bit for bit in
        every shape."""
        self._check(self.lib.avbd_batch_set_launch(self.handle, collide_threads, solve_blocks, rows_per_lane, world_threads))

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.avbd_batch_stream(self.handle, ctypes.byref(s)))
        return s.value or 0

    # --- readbacks ---
    def read_bodies(self, w: int) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_batch_read_bodies(self.handle, w, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=BODY_DTYPE)
        self._check(self.lib.avbd_batch_read_bodies(self.handle, w, ptr(out), n.value, ctypes.byref(n)))
        return out

    def read_joints(self, w: int):
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_batch_read_joints(self.handle, w, None, None, 0, ctypes.byref(n)))
        recs = np.zeros(n.value, dtype=JOINT_DTYPE)
        info = np.zeros(n.value, dtype=INFO_DTYPE)
        self._check(self.lib.avbd_batch_read_joints(self.handle, w, ptr(recs), ptr(info), n.value, ctypes.byref(n)))
        return recs, info

    def read_colors(self, w: int) -> np.ndarray:
        n = ctypes.c_uint32()
        self._check(self.lib.avbd_batch_read_colors(self.handle, w, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, dtype=np.uint32)
        self._check(self.lib.avbd_batch_read_colors(self.handle, w, uptr(out), n.value, ctypes.byref(n)))
        return out

    def read_counters(self, w: int) -> dict:
        c = Counters()
        self._check(self.lib.avbd_batch_read_counters(self.handle, w, ctypes.byref(c)))
        return c.as_dict()

    def read_all_bodies_into(self, out: np.ndarray, sync: bool = True):
        """Every world's bodies, world w at its first_body, into caller memory (pinned for overlap)."""
        self._check(self.lib.avbd_batch_read_all_bodies_async(self.handle, ptr(out), len(out)))
        if sync:
            self.synchronize()

    def write_all_bodies_async(self, records: np.ndarray):
        self._check(self.lib.avbd_batch_write_all_bodies_async(self.handle, ptr(records), len(records)))

    def record_start(self, steps: int, points_per_body: int = 0):
        """Record the contact structure of the next `steps` steps for the adjoint (Adjoint.from_batch)."""
        self._check(self.lib.avbd_batch_record_start(self.handle, steps, points_per_body))

    def record_status(self) -> dict:
        st, pr = ctypes.c_uint32(), ctypes.c_uint32()
        m, p = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self.lib.avbd_batch_record_status(self.handle, ctypes.byref(st), ctypes.byref(m), ctypes.byref(p), ctypes.byref(pr)))
        return {'steps': st.value, 'manifolds': m.value, 'points': p.value, 'problems': pr.value}
