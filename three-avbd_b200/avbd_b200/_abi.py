"""ctypes view of include/avbd.h: loads libavbd_cuda.so and declares every entry point.

The record dtypes are byte-for-byte the C structs (and the reference's GPU records: a body is 40
floats, src/avbd3d/gpu/layout.ts:8-59; a joint 40 floats, layout.ts:77-110; a manifold 8 words and a
contact 16 words, layout.ts:118-127). There is no CPU fallback: if the library or a B200 is missing,
the solver raises.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libavbd_cuda.so')

AVBD_OK = 0
AVBD_ERR_INVALID = -1
AVBD_ERR_CAPACITY = -2
AVBD_ERR_CUDA = -3
AVBD_ERR_TIMEOUT = -4
AVBD_ERR_NO_DEVICE = -5

SHAPE_BOX, SHAPE_SPHERE, SHAPE_SAIL = 0, 1, 2
T_NONE, T_JOINT, T_SPRING = 0, 1, 2
FLAG_MATCH_NEAREST, FLAG_FACE_BIAS, FLAG_REUSE_CONTACTS, FLAG_START_AT_REST, FLAG_MASS_PENALTY = 1, 2, 4, 8, 16
STICK_BIT = 0x80000000
NO_COLOR = 255
PENDING = 256
MAX_COLORS = 64
BIG = np.float32(3.0e38)

BODY_DTYPE = np.dtype([
    ('pos', '<f4', 3), ('friction', '<f4'), ('rot', '<f4', 4), ('initial_pos', '<f4', 3), ('flags', '<f4'),
    ('initial_rot', '<f4', 4), ('size', '<f4', 3), ('mass', '<f4'), ('moment', '<f4', 3), ('radius', '<f4'),
    ('inertial_pos', '<f4', 3), ('moved_step', '<f4'), ('inertial_rot', '<f4', 4), ('vel', '<f4', 3), ('prev_up_vel', '<f4'),
    ('ang_vel', '<f4', 3), ('shape', '<f4'),
])
JOINT_DTYPE = np.dtype([
    ('pen_lin', '<f4', 3), ('stiffness_lin', '<f4'), ('pen_ang', '<f4', 3), ('stiffness_ang', '<f4'),
    ('lam_lin', '<f4', 3), ('fracture', '<f4'), ('lam_ang', '<f4', 3), ('torque_arm', '<f4'),
    ('c0_lin', '<f4', 4), ('c0_ang', '<f4', 3), ('yield_force', '<f4'), ('r_a', '<f4', 3), ('spring_rest', '<f4'),
    ('r_b', '<f4', 3), ('break_bend', '<f4'), ('rest', '<f4', 4), ('rest_start', '<f4', 4),
])
INFO_DTYPE = np.dtype([('type', '<i4'), ('a', '<i4'), ('b', '<i4'), ('meta', '<i4')])
MANIFOLD_DTYPE = np.dtype([('a', '<u4'), ('b', '<u4'), ('first', '<u4'), ('count', '<u4'), ('normal', '<f4', 3), ('friction', '<f4')])
CONTACT_DTYPE = np.dtype([
    ('r_a', '<f4', 3), ('key', '<u4'), ('r_b', '<f4', 3), ('c0_n', '<f4'), ('pen', '<f4', 3), ('c0_t1', '<f4'),
    ('lam', '<f4', 3), ('c0_t2', '<f4'),
])
PUSH_DTYPE = np.dtype([('body', '<u4'), ('lin', '<f4', 3), ('off_lin', '<f4', 3), ('moment', '<f4', 3)])
EVENT_DTYPE = np.dtype([('kind', '<u4'), ('a', '<u4'), ('b', '<u4'), ('step', '<u4'), ('point', '<f4', 3), ('impulse', '<f4'),
                        ('normal', '<f4', 3), ('pad', '<f4')])
RAY_DTYPE = np.dtype([('origin', '<f4', 3), ('max_distance', '<f4'), ('direction', '<f4', 3), ('pad', '<f4')])
HIT_DTYPE = np.dtype([('body', '<i4'), ('distance', '<f4'), ('point', '<f4', 3), ('normal', '<f4', 3)])
CONTACT_BEGIN, CONTACT_END = 1, 2
RAY_MAX, RAY_MAX_IGNORED = 65535, 16
STEP_STATS_DTYPE = np.dtype([('collision_ms', '<f4'), ('solve_ms', '<f4')] + [(n, '<u4') for n in (
    'pairs', 'contacts', 'manifolds', 'adjacency', 'incidences', 'dynamic_bodies', 'colors', 'rounds', 'launches', 'error')])
assert BODY_DTYPE.itemsize == 160 and JOINT_DTYPE.itemsize == 160 and MANIFOLD_DTYPE.itemsize == 32 and CONTACT_DTYPE.itemsize == 64
assert PUSH_DTYPE.itemsize == 40 and EVENT_DTYPE.itemsize == 48 and RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 32


class Params(ctypes.Structure):
    _fields_ = [('dt', ctypes.c_float), ('gravity', ctypes.c_float), ('alpha', ctypes.c_float), ('beta_lin', ctypes.c_float),
                ('beta_ang', ctypes.c_float), ('gamma', ctypes.c_float), ('contact_margin', ctypes.c_float), ('iterations', ctypes.c_int32),
                ('flags', ctypes.c_uint32), ('up', ctypes.c_float * 3),
                ('wind_speed', ctypes.c_float), ('wind_angle', ctypes.c_float), ('wind_gust', ctypes.c_float), ('wind_pressure', ctypes.c_float)]


class Config(ctypes.Structure):
    _fields_ = [('body_capacity', ctypes.c_uint32), ('joint_capacity', ctypes.c_uint32), ('pair_capacity', ctypes.c_uint32), ('device', ctypes.c_int32)]


class Counters(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ('pairs', 'contacts', 'manifolds', 'overflow', 'clashes', 'colors', 'rounds', 'error', 'steps',
                                                'pair_capacity', 'graphs', 'launches')]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if not n.startswith('reserved')}


class HullProps(ctypes.Structure):
    _fields_ = [('volume', ctypes.c_double), ('moments', ctypes.c_double * 3), ('size', ctypes.c_double * 3), ('radius', ctypes.c_double),
                ('center', ctypes.c_double * 3), ('rotation', ctypes.c_double * 4), ('vertices', ctypes.c_uint32), ('faces', ctypes.c_uint32),
                ('edges', ctypes.c_uint32)]


SHAPE_HULL = 3
MAX_HULL_VERTICES = 32


class BodyView(ctypes.Structure):
    _fields_ = [('fields', ctypes.c_void_p * 10), ('count', ctypes.c_uint32), ('capacity', ctypes.c_uint32)]


class ContactView(ctypes.Structure):
    _fields_ = [('pairs', ctypes.c_void_p), ('normals', ctypes.c_void_p), ('points', ctypes.c_void_p), ('counters', ctypes.c_void_p),
                ('count_word', ctypes.c_uint32), ('pair_capacity', ctypes.c_uint32)]


class BatchConfig(ctypes.Structure):
    _fields_ = [('world_capacity', ctypes.c_uint32), ('body_capacity', ctypes.c_uint32), ('joint_capacity', ctypes.c_uint32),
                ('pairs_per_body', ctypes.c_uint32), ('device', ctypes.c_int32)]


class StepOptions(ctypes.Structure):
    _fields_ = [('reuse_manifolds', ctypes.c_uint32)]


class BatchWorld(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ('first_body', 'bodies', 'first_joint', 'joints', 'pair_capacity', 'fixed_colors')]


class BatchStatus(ctypes.Structure):
    _fields_ = [('worlds', ctypes.c_uint32), ('bodies', ctypes.c_uint32), ('joints', ctypes.c_uint32), ('steps', ctypes.c_uint32),
                ('pair_slots', ctypes.c_uint64), ('relayouts', ctypes.c_uint32), ('collide_threads', ctypes.c_uint32),
                ('collide_blocks', ctypes.c_uint32), ('solve_blocks', ctypes.c_uint32), ('graphs', ctypes.c_uint32),
                ('rows_per_lane', ctypes.c_uint32), ('world_threads', ctypes.c_uint32)]


NOALLOC_MAX_BODIES = 4096
NOALLOC_MAX_PAIRS = 32768
TUNE_CANDIDATES = 16
BATCH_MAX_WORLD_BODIES = 4096


class BatchTuning(ctypes.Structure):
    _fields_ = [('candidates', ctypes.c_uint32), ('candidate_threads', ctypes.c_uint32 * TUNE_CANDIDATES),
                ('candidate_solve_blocks', ctypes.c_uint32 * TUNE_CANDIDATES), ('candidate_rows_per_lane', ctypes.c_uint32 * TUNE_CANDIDATES),
                ('candidate_ms', ctypes.c_float * TUNE_CANDIDATES), ('collide_threads', ctypes.c_uint32), ('solve_blocks', ctypes.c_uint32),
                ('rows_per_lane', ctypes.c_uint32), ('ms_per_step', ctypes.c_float), ('steps_taken', ctypes.c_uint32),
                ('candidate_world_threads', ctypes.c_uint32 * TUNE_CANDIDATES), ('world_threads', ctypes.c_uint32)]


# Every function include/avbd.h declares, with its argument types (the C-ABI symbol table)
P, U, I, VP = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p
PU = ctypes.POINTER(ctypes.c_uint32)
SIGNATURES = {
    'avbd_abi_version': ([], I),
    'avbd_device_info': ([I, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int)], I),
    'avbd_world_create': ([ctypes.POINTER(Config), ctypes.POINTER(P)], I),
    'avbd_world_destroy': ([P], I),
    'avbd_last_error': ([P], ctypes.c_char_p),
    'avbd_set_params': ([P, ctypes.POINTER(Params)], I),
    'avbd_get_params': ([P, ctypes.POINTER(Params)], I),
    'avbd_default_params': ([ctypes.POINTER(Params)], I),
    'avbd_world_params': ([ctypes.POINTER(Params)], I),
    'avbd_add_bodies': ([P, VP, U, PU], I),
    'avbd_write_bodies': ([P, U, VP, U, I], I),
    'avbd_write_bodies_at': ([P, PU, VP, U], I),
    'avbd_add_joints': ([P, VP, VP, U, PU], I),
    'avbd_write_joints': ([P, U, VP, VP, U], I),
    'avbd_release_joints': ([P, PU, U], I),
    'avbd_broadphase_radii': ([ctypes.POINTER(ctypes.c_double), U, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)], I),
    'avbd_append_joints': ([P, VP, VP, U, PU], I),
    'avbd_disable_joints': ([P, PU, U], I),
    'avbd_add_world_joint': ([P, U, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), PU], I),
    'avbd_set_world_anchor': ([P, U, ctypes.POINTER(ctypes.c_float)], I),
    'avbd_body_storage': ([P, ctypes.POINTER(BodyView)], I),
    'avbd_contact_storage': ([P, U, ctypes.POINTER(ContactView)], I),
    'avbd_add_ignore_pairs': ([P, PU, U], I),
    'avbd_set_filters': ([P, U, PU, U], I),
    'avbd_set_filters_at': ([P, PU, PU, PU, U], I),
    'avbd_seed_contacts': ([P, VP, U, VP, U], I),
    'avbd_set_fixed_colors': ([P, PU, U], I),
    'avbd_step': ([P, I], I),
    'avbd_step_with': ([P, I, ctypes.POINTER(StepOptions)], I),
    'avbd_apply_pushes': ([P, VP, U], I),
    'avbd_contact_watch_create': ([P, U, U, ctypes.POINTER(P)], I),
    'avbd_contact_watch_destroy': ([P], I),
    'avbd_contact_watch_last_error': ([P], ctypes.c_char_p),
    'avbd_contact_watch_set': ([P, PU, PU, PU, U], I),
    'avbd_contact_watch_run': ([P, U, ctypes.c_float], I),
    'avbd_contact_watch_read': ([P, VP, U, PU, PU, PU], I),
    'avbd_raycast': ([P, VP, U, PU, U, U, VP], I),
    'avbd_pose_capture_create': ([P, PU, U, U, ctypes.POINTER(P)], I),
    'avbd_pose_capture_frame': ([P], I),
    'avbd_pose_capture_read': ([P, PU, ctypes.POINTER(ctypes.c_float), U, PU, PU], I),
    'avbd_pose_capture_reset': ([P], I),
    'avbd_pose_capture_destroy': ([P], I),
    'avbd_read_reuse_state': ([P, ctypes.POINTER(ctypes.c_float), U, PU, PU, U, PU], I),
    'avbd_synchronize': ([P], I),
    'avbd_read_bodies': ([P, VP, U, PU], I),
    'avbd_read_joints': ([P, VP, VP, U, PU], I),
    'avbd_read_contacts': ([P, VP, U, PU, VP, U, PU], I),
    'avbd_read_pairs': ([P, PU, U, PU], I),
    'avbd_read_colors': ([P, PU, U, PU], I),
    'avbd_read_counters': ([P, ctypes.POINTER(Counters)], I),
    'avbd_read_bodies_async': ([P, VP, U], I),
    'avbd_enable_step_stats': ([P, U], I),
    'avbd_read_step_stats': ([P, VP, U, PU], I),
    'avbd_world_stream': ([P, ctypes.POINTER(ctypes.c_void_p)], I),
    'avbd_use_graphs': ([P, I], I),
    'avbd_set_solve_blocks': ([P, I], I),
    'avbd_read_phase_clocks': ([P, ctypes.POINTER(ctypes.c_double), U, PU], I),
    'avbd_write_bodies_async': ([P, U, VP, U], I),
    'avbd_hull_build': ([VP, U, PU, U, PU, ctypes.POINTER(HullProps)], I),
    'avbd_add_hull': ([P, PU, U, PU], I),
    'avbd_find_pairs_noalloc': ([VP, U, PU, PU, U, PU, VP], I),
    'avbd_adjoint_create': ([VP, ctypes.POINTER(P)], I),
    'avbd_adjoint_destroy': ([P], I),
    'avbd_adjoint_last_error': ([P], ctypes.c_char_p),
    'avbd_adjoint_set_target': ([P, ctypes.POINTER(ctypes.c_double)], I),
    'avbd_adjoint_forward': ([P] + [ctypes.POINTER(ctypes.c_double)] * 3, I),
    'avbd_adjoint_backward': ([P] + [ctypes.POINTER(ctypes.c_double)] * 3, I),
    'avbd_set_body_aux': ([P, VP, U, VP, VP, VP], I),
    'avbd_read_body_aux': ([P, U, VP, U], I),
    'avbd_set_lifecycle': ([P, U, U], I),
    'avbd_release_hull': ([P, U], I),
    'avbd_hull_storage': ([P, ctypes.POINTER(U), ctypes.POINTER(U), ctypes.POINTER(U)], I),
    'avbd_adjoint_create_from_batch': ([P, ctypes.c_uint32, ctypes.POINTER(P)], I),
    'avbd_adjoint_nominal': ([P, ctypes.POINTER(ctypes.c_double)], I),
    'avbd_adjoint_read_recording': ([P] + [VP] * 10, I),
    'avbd_adjoint_info': ([P] + [ctypes.POINTER(ctypes.c_uint32)] * 4 + [ctypes.POINTER(ctypes.c_uint64)] * 2, I),
    'avbd_batch_record_start': ([P, ctypes.c_uint32, ctypes.c_uint32], I),
    'avbd_batch_record_status': ([P, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                  ctypes.POINTER(ctypes.c_uint32)], I),
    'avbd_batch_create': ([ctypes.POINTER(BatchConfig), ctypes.POINTER(P)], I),
    'avbd_batch_destroy': ([P], I),
    'avbd_batch_last_error': ([P], ctypes.c_char_p),
    'avbd_batch_set_params': ([P, ctypes.POINTER(Params)], I),
    'avbd_batch_add_world': ([P, VP, U, VP, VP, U, PU, U, PU], I),
    'avbd_batch_add_world_from': ([P, P, PU], I),
    'avbd_batch_world_info': ([P, U, ctypes.POINTER(BatchWorld)], I),
    'avbd_batch_step': ([P, I], I),
    'avbd_batch_synchronize': ([P], I),
    'avbd_batch_read_bodies': ([P, U, VP, U, PU], I),
    'avbd_batch_read_joints': ([P, U, VP, VP, U, PU], I),
    'avbd_batch_read_colors': ([P, U, PU, U, PU], I),
    'avbd_batch_read_counters': ([P, U, ctypes.POINTER(Counters)], I),
    'avbd_batch_read_all_bodies_async': ([P, VP, U], I),
    'avbd_batch_write_all_bodies_async': ([P, VP, U], I),
    'avbd_batch_use_graphs': ([P, I], I),
    'avbd_batch_stream': ([P, ctypes.POINTER(ctypes.c_void_p)], I),
    'avbd_batch_tune': ([P, I, ctypes.POINTER(BatchTuning)], I),
    'avbd_batch_info': ([P, ctypes.POINTER(BatchStatus)], I),
    'avbd_batch_set_launch': ([P, U, U, U, U], I),
}

_lib = None


def load(path: str = LIB_PATH):
    """The CUDA library, with every declared symbol bound. Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f'{path} is missing: build it with three-avbd_b200/build.py (there is no CPU fallback)')
    lib = ctypes.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


class AvbdError(RuntimeError):
    """A negative status of the C ABI (the reference throws `Error` before any state change)."""

    def __init__(self, code: int, message: str):
        super().__init__(f'avbd error {code}: {message}')
        self.code = code


class StorageCapacityError(AvbdError):
    """AVBD_ERR_CAPACITY: a fixed capacity would be passed (src/lib/storage-budget.ts:32-42)."""


class DeviceError(AvbdError):
    """AVBD_ERR_CUDA / AVBD_ERR_NO_DEVICE: the device failed or is missing (World's gpuError, world.ts:874-877)."""


class DeviceTimeout(AvbdError):
    """AVBD_ERR_TIMEOUT: a bounded device wait gave up; the step's results are not valid."""


def error(code: int, message: str) -> AvbdError:
    """The exception for a C-ABI status."""
    kind = {AVBD_ERR_CAPACITY: StorageCapacityError, AVBD_ERR_CUDA: DeviceError, AVBD_ERR_NO_DEVICE: DeviceError,
            AVBD_ERR_TIMEOUT: DeviceTimeout}.get(code, AvbdError)
    return kind(code, message)


def ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def uptr(a: np.ndarray):
    return a.ctypes.data_as(PU)
