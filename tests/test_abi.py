"""The C-ABI library loads and exports every symbol include/avbd.h declares (no GPU needed)."""

import ctypes
import os
import re

import pytest

import avbd_b200
from avbd_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, 'include', 'avbd.h')).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(avbd_[a-z0-9_]+)\s*\(', text)))


def test_every_declared_symbol_is_exported():
    lib = avbd_b200.load()
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), f'{name} is declared in avbd.h but not exported'
        assert name in _abi.SIGNATURES, f'{name} has no ctypes signature'


def test_record_layouts_match_the_reference():
    # layout.ts:15 BODY_FLOATS = 40, :77 JOINT_FLOATS = 40, :118 MANIFOLD_WORDS = 8, :123 CONTACT_WORDS = 16
    assert _abi.BODY_DTYPE.itemsize == 40 * 4
    assert _abi.JOINT_DTYPE.itemsize == 40 * 4
    assert _abi.MANIFOLD_DTYPE.itemsize == 8 * 4
    assert _abi.CONTACT_DTYPE.itemsize == 16 * 4
    assert ctypes.sizeof(_abi.Params) == 16 * 4


def test_defaults_and_invalid_arguments_without_a_device():
    lib = avbd_b200.load()
    p = _abi.Params()
    assert lib.avbd_default_params(ctypes.byref(p)) == 0
    assert abs(p.dt - 1 / 60) < 1e-7 and p.iterations == 10 and p.gravity == -10.0 and tuple(p.up) == (0.0, 0.0, 1.0)
    assert p.wind_pressure == 0.0 and p.wind_speed == 0.0  # no air: sails fall as the CPU solver's boxes
    assert lib.avbd_abi_version() == 3
    assert lib.avbd_world_create(None, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_world_destroy(None) == 0
    assert lib.avbd_step(None, 1) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_add_world_joint(None, 0, None, None, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_append_joints(None, None, None, 0, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_disable_joints(None, None, 0) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_set_world_anchor(None, 0, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_body_storage(None, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_contact_storage(None, 0, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_step_with(None, 1, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_read_reuse_state(None, None, 0, None, None, 0, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_apply_pushes(None, None, 0) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_contact_watch_create(None, 16, 16, None) == _abi.AVBD_ERR_INVALID
    assert lib.avbd_contact_watch_destroy(None) == 0
    assert lib.avbd_raycast(None, None, 0, None, 0, 0, None) == _abi.AVBD_ERR_INVALID


def test_world_params_are_the_reference_production_defaults():
    """avbd_world_params (gpuParams3D(), gpu/solver.ts:216-230): every GPU-only rule on, up = +y;
    avbd_default_params keeps the parity setting (rules off, up = +z)."""
    lib = avbd_b200.load()
    p = _abi.Params()
    assert lib.avbd_world_params(ctypes.byref(p)) == 0
    rules = _abi.FLAG_MATCH_NEAREST | _abi.FLAG_FACE_BIAS | _abi.FLAG_REUSE_CONTACTS | _abi.FLAG_START_AT_REST | _abi.FLAG_MASS_PENALTY
    assert p.flags == rules and tuple(p.up) == (0.0, 1.0, 0.0) and abs(p.contact_margin - 0.01) < 1e-9 and p.iterations == 10
    # calm air (gpu/solver.ts:226-229): no wind, gusts 0.4 of it, pressure coefficient 0.72
    assert (p.wind_speed, p.wind_angle) == (0.0, 0.0) and abs(p.wind_gust - 0.4) < 1e-7 and abs(p.wind_pressure - 0.72) < 1e-7


def test_query_record_layouts():
    assert _abi.PUSH_DTYPE.itemsize == 40 and _abi.EVENT_DTYPE.itemsize == 48
    assert _abi.RAY_DTYPE.itemsize == 32 and _abi.HIT_DTYPE.itemsize == 32
    assert ctypes.sizeof(_abi.BatchTuning) == 4 + 4 * 16 * 5 + 4 * 6
    assert ctypes.sizeof(_abi.BatchStatus) == 56  # 4 words, a 64-bit count, 7 words, padded to 8 bytes


def test_create_fails_loudly_without_a_b200():
    """There is no CPU fallback: without a B200 the world cannot be made."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip('a GPU is present')
    with pytest.raises(avbd_b200.DeviceError):
        avbd_b200.CudaSolver3D(avbd_b200.scenes.demo_scene('Ground'))


def test_statuses_map_to_the_reference_errors():
    e = _abi.error(_abi.AVBD_ERR_CAPACITY, 'body capacity 4 reached')
    assert isinstance(e, avbd_b200.StorageCapacityError) and isinstance(e, avbd_b200.AvbdError) and e.code == _abi.AVBD_ERR_CAPACITY
    assert isinstance(_abi.error(_abi.AVBD_ERR_NO_DEVICE, ''), avbd_b200.DeviceError)
    assert isinstance(_abi.error(_abi.AVBD_ERR_CUDA, ''), avbd_b200.DeviceError)
    assert isinstance(_abi.error(_abi.AVBD_ERR_TIMEOUT, ''), avbd_b200.DeviceTimeout)
    e = _abi.error(_abi.AVBD_ERR_INVALID, 'joint 0: NaN')
    assert type(e) is avbd_b200.AvbdError and 'joint 0: NaN' in str(e)
