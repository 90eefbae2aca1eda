"""The pose cache on-disk format (src/bake/pose-cache.ts, schema `three-avbd.pose-cache/v0-draft`): a
canonical compact-JSON manifest plus little-endian binary chunks, each frame a u32 step, seven f32 per
body slot (position, then quaternion x y z w) and a CRC-32 chained from its chunk header's. The byte
layout, the manifest's key order and number spelling, the limits and the checks are the reference's,
so that caches written here read there and the reverse; the frames themselves come from a CUDA world
through PoseCapture (avbd_pose_capture_*), which gathers them on the device each sampled step.

Errors raise PoseCacheError with the reference's codes ('argument', 'schema', 'manifest', 'budget',
'chunk', 'data'); arrays passed in are never kept or changed."""

from __future__ import annotations

import json
import math
import re
import struct
import zlib
from dataclasses import dataclass, field

import numpy as np

POSE_CACHE_SCHEMA = 'three-avbd.pose-cache/v0-draft'
POSE_CACHE_CHUNK_REVISION = 1
POSE_CACHE_CONVENTIONS = {'length': 'metre', 'time': 'second', 'handedness': 'right', 'up': '+y', 'rotation': 'quaternion-xyzw',
                          'pose': 'position-xyz-then-rotation-xyzw', 'byteOrder': 'little', 'floatFormat': 'float32'}
POSE_FLOATS = 7
POSE_SLOT_BYTES = POSE_FLOATS * 4
CHUNK_HEADER_BYTES = 36
CHUNK_MAGIC = b'TAPC'

DEFAULT_LIMITS = {'maxBodies': 4096, 'maxFrames': 36_000, 'maxChunks': 1024, 'maxChunkBytes': 16 * 1024 * 1024,
                  'maxTotalBytes': 256 * 1024 * 1024, 'maxManifestBytes': 1024 * 1024}
HARD_LIMITS = {'maxBodies': 65_536, 'maxFrames': 1_000_000, 'maxChunks': 65_536, 'maxChunkBytes': 64 * 1024 * 1024,
               'maxTotalBytes': 1024 * 1024 * 1024, 'maxManifestBytes': 16 * 1024 * 1024}
VALUE_LIMITS = {'maxCoordinate': 1e6, 'maxSize': 1e3, 'maxDt': 1, 'quaternionTolerance': 1e-3, 'maxId': 0x7FFFFFFF,
                'provenanceKeys': 32, 'provenanceStringLength': 256}
TERMINATIONS = ('complete', 'cancelled', 'budget', 'recovered')


def pose_frame_bytes(bodies: int) -> int:
    """Bytes of one frame record: u32 step, one slot per body, u32 CRC-32 of the step and slots."""
    return 8 + POSE_SLOT_BYTES * bodies


class PoseCacheError(Exception):
    def __init__(self, code: str, message: str):
        super().__init__(message)
        self.code = code


def _fail(code: str, message: str):
    raise PoseCacheError(code, message)


def crc32(data, start: int = 0, end: int | None = None, previous: int = 0) -> int:
    """CRC-32 (IEEE, as zlib) of data[start:end], continuing a finished prior CRC when given."""
    b = memoryview(bytes(data) if not isinstance(data, (bytes, bytearray, memoryview)) else data)
    return zlib.crc32(b[start:end], previous) & 0xFFFFFFFF


@dataclass
class PoseCacheBody:
    id: int
    shape: str          # 'box' | 'sphere'
    size: list          # full widths (m); a sphere's diameter on every axis
    fixed: bool
    first_frame: int    # alive in frames [first_frame, end_frame)
    end_frame: int


@dataclass
class PoseCache:
    cache_id: int
    dt: float
    bodies: list                 # PoseCacheBody
    steps: np.ndarray            # uint32, strictly increasing
    poses: np.ndarray            # float32, frames x bodies x 7; +0 outside a body's lifetime
    termination: str = 'complete'
    provenance: dict | None = None


@dataclass
class PoseCacheRecovery:
    cache: PoseCache | None
    complete: bool
    declared_frames: int
    recovered_frames: int
    omitted_body_ids: list = field(default_factory=list)
    problem: dict | None = None


def resolve_limits(partial: dict | None = None) -> dict:
    """Caller limits checked against the hard ceilings, completed from the defaults."""
    out = dict(DEFAULT_LIMITS)
    if partial is None:
        return out
    if not isinstance(partial, dict):
        _fail('argument', 'limits must be a plain object')
    for k, v in partial.items():
        if k not in HARD_LIMITS:
            _fail('argument', f'limits: unknown limit "{str(k)[:40]}"')
        if not _is_int(v, 1, HARD_LIMITS[k]):
            _fail('argument', f'limits.{k} must be an integer from 1 to {HARD_LIMITS[k]}')
        out[k] = v
    return out


def _is_int(v, lo, hi) -> bool:
    return isinstance(v, int) and not isinstance(v, bool) and lo <= v <= hi


def _finite(v) -> bool:
    return isinstance(v, (int, float)) and not isinstance(v, bool) and math.isfinite(v)


# ---- JSON number and text spelling (ECMAScript Number::toString and JSON.stringify) --------------

def js_number(x) -> str:
    """A number spelled as JSON.stringify spells it: the shortest round-trip digits, in plain notation
    for decimal exponents from -6 to 20 and exponent notation (1e+21, 1.5e-7) outside them."""
    if isinstance(x, bool):
        raise TypeError('not a number')
    if isinstance(x, int):
        return str(x)
    x = float(x)
    if x == 0:
        return '0'
    if x < 0:
        return '-' + js_number(-x)
    mant, _, exp = repr(x).partition('e')
    e10 = int(exp) if exp else 0
    whole, _, frac = mant.partition('.')
    digits = (whole + frac).lstrip('0')
    # position of the decimal point relative to the digit string: value = 0.digits x 10^n
    n = len(whole.lstrip('0')) + e10 if whole.strip('0') else e10 - (len(frac) - len(frac.lstrip('0')))
    digits = digits.rstrip('0') or '0'
    k = len(digits)
    if k <= n <= 21:
        return digits + '0' * (n - k)
    if 0 < n <= 21:
        return digits[:n] + '.' + digits[n:]
    if -6 < n <= 0:
        return '0.' + '0' * (-n) + digits
    e = n - 1
    sign = '+' if e >= 0 else '-'
    return (digits[0] + ('.' + digits[1:] if k > 1 else '')) + 'e' + sign + str(abs(e))


def _js_value(v) -> str:
    if v is None:
        return 'null'
    if v is True:
        return 'true'
    if v is False:
        return 'false'
    if isinstance(v, (int, float)):
        return js_number(v)
    if isinstance(v, str):
        return json.dumps(v, ensure_ascii=True)
    if isinstance(v, (list, tuple)):
        return '[' + ','.join(_js_value(x) for x in v) + ']'
    if isinstance(v, dict):
        return '{' + ','.join(json.dumps(str(k)) + ':' + _js_value(x) for k, x in v.items()) + '}'
    raise TypeError(f'cannot spell {type(v).__name__}')


# ---- bodies, provenance, values -----------------------------------------------------------------

_BODY_KEYS = ('id', 'shape', 'size', 'fixed', 'firstFrame', 'endFrame')


def _body_from(b, at: str, frame_count: int, code: str) -> PoseCacheBody:
    """One body table entry (a PoseCacheBody or the manifest's dict) checked against `frame_count`."""
    if isinstance(b, PoseCacheBody):
        d = {'id': b.id, 'shape': b.shape, 'size': b.size, 'fixed': b.fixed, 'firstFrame': b.first_frame, 'endFrame': b.end_frame}
    elif isinstance(b, dict):
        d = b
        for k in d:
            if k not in _BODY_KEYS:
                _fail(code, f'{at}: unknown field "{str(k)[:40]}"')
    else:
        _fail(code, f'{at}: expected an object')
    bid, shape, size, fixed, first, end = (d.get(k) for k in _BODY_KEYS)
    if not _is_int(bid, 1, VALUE_LIMITS['maxId']):
        _fail(code, f'{at}: id must be an integer from 1 to {VALUE_LIMITS["maxId"]}')
    if shape not in ('box', 'sphere'):
        _fail(code, f'{at}: shape must be "box" or "sphere" (nothing else is cached yet)')
    if not isinstance(size, (list, tuple)) or len(size) != 3 or not all(_finite(v) and 0 < v <= VALUE_LIMITS['maxSize'] for v in size):
        _fail(code, f'{at}: size must be three numbers above 0 and at most {VALUE_LIMITS["maxSize"]}')
    if shape == 'sphere' and not (size[0] == size[1] == size[2]):
        _fail(code, f"{at}: a sphere's size is its diameter on all three axes")
    if not isinstance(fixed, bool):
        _fail(code, f'{at}: fixed must be true or false')
    if not _is_int(first, 0, frame_count - 1):
        _fail(code, f'{at}: firstFrame must be a frame index below {frame_count}')
    if not _is_int(end, first + 1, frame_count):
        _fail(code, f'{at}: endFrame must be above firstFrame and at most {frame_count}')
    return PoseCacheBody(bid, shape, [size[0], size[1], size[2]], fixed, first, end)


def _bodies_from(lst, frame_count: int, limits: dict, code: str) -> list:
    if not isinstance(lst, (list, tuple)) or len(lst) < 1:
        _fail(code, 'bodies must be a non-empty list')
    if len(lst) > limits['maxBodies']:
        _fail('budget', f'{len(lst)} bodies exceed the limit of {limits["maxBodies"]}')
    seen, out = set(), []
    for i, b in enumerate(lst):
        body = _body_from(b, f'bodies[{i}]', frame_count, code)
        if body.id in seen:
            _fail(code, f'bodies[{i}]: duplicate id {body.id}')
        seen.add(body.id)
        out.append(body)
    return out


_PROVENANCE_KEY = re.compile(r'^[A-Za-z][A-Za-z0-9_.-]{0,63}$')
_PROVENANCE_TEXT = re.compile(r'^[\x20-\x7e]*$')


def _provenance_from(v, code: str):
    """A flat, bounded record of printable-ASCII strings, finite numbers, booleans and nulls; None: none."""
    if v is None:
        return None
    if not isinstance(v, dict):
        _fail(code, 'provenance must be an object when present')
    if len(v) > VALUE_LIMITS['provenanceKeys']:
        _fail(code, f'provenance may hold at most {VALUE_LIMITS["provenanceKeys"]} entries')
    out = {}
    for k, x in v.items():
        if not isinstance(k, str) or not _PROVENANCE_KEY.match(k):
            _fail(code, 'provenance: keys must start with a letter and use letters, digits, "_", "." or "-" (64 at most)')
        ok_text = isinstance(x, str) and len(x) <= VALUE_LIMITS['provenanceStringLength'] and _PROVENANCE_TEXT.match(x)
        if not (ok_text or _finite(x) or isinstance(x, bool) or x is None):
            _fail(code, f'provenance.{k}: expected printable ASCII text ({VALUE_LIMITS["provenanceStringLength"]} at most), a finite number, a boolean or null')
        out[k] = x
    return out


def pose_body_table_crc32(dt: float, bodies: list, cache_id: int) -> int:
    """CRC-32 over a fixed little-endian encoding of cache_id, dt and each body's id, shape (1 box,
    2 sphere), fixed flag and size (lifetimes excluded)."""
    buf = bytearray(16 + 30 * len(bodies))
    struct.pack_into('<IId', buf, 0, cache_id, len(bodies), float(dt))
    for i, b in enumerate(bodies):
        struct.pack_into('<IBBddd', buf, 16 + 30 * i, b.id, 1 if b.shape == 'box' else 2, 1 if b.fixed else 0, *(float(s) for s in b.size))
    return crc32(buf)


def _slot_problem(p: np.ndarray, alive: bool):
    """Why a slot is wrong: alive, finite bounded position and unit quaternion; not alive, +0 everywhere."""
    if not alive:
        if np.any(p.view(np.uint32) != 0):
            return 'a slot outside its lifetime must be all +0'
        return None
    if not np.all(np.abs(p[:3].astype(np.float64)) <= VALUE_LIMITS['maxCoordinate']):
        return f'position must be finite and within ±{js_number(VALUE_LIMITS["maxCoordinate"])} m'
    if not np.all(np.isfinite(p[3:7])):
        return 'rotation must be finite'
    length = math.hypot(*(float(x) for x in p[3:7]))
    if not abs(length - 1) <= VALUE_LIMITS['quaternionTolerance']:
        return f'rotation must be a unit quaternion (length {length:.4g})'
    return None


def _frame_problem(frame_poses: np.ndarray, bodies: list, frame: int):
    for i, b in enumerate(bodies):
        problem = _slot_problem(frame_poses[i], b.first_frame <= frame < b.end_frame)
        if problem:
            return f'frame {frame}, body {b.id}: {problem}'
    return None


# ---- manifest -----------------------------------------------------------------------------------

_TOP_KEYS = ('schema', 'conventions', 'cacheId', 'termination', 'dt', 'bodyTableCrc32', 'bodies', 'frameCount', 'chunks', 'budget', 'provenance')
_CHUNK_KEYS = ('index', 'firstFrame', 'frameCount', 'byteLength')
_BUDGET_KEYS = ('maxBodies', 'maxFrames', 'maxBytes')


@dataclass
class PoseCacheManifest:
    cache_id: int
    termination: str
    dt: float
    body_table_crc32: int
    bodies: list
    frame_count: int
    chunks: list        # dicts: index, firstFrame, frameCount, byteLength
    budget: dict        # maxBodies, maxFrames, maxBytes
    provenance: dict | None


def _serialize_manifest(m: PoseCacheManifest) -> str:
    """The one accepted text: compact JSON in the fixed key order, JavaScript's number spelling."""
    value = {
        'schema': POSE_CACHE_SCHEMA, 'conventions': POSE_CACHE_CONVENTIONS, 'cacheId': m.cache_id, 'termination': m.termination, 'dt': m.dt,
        'bodyTableCrc32': m.body_table_crc32,
        'bodies': [{'id': b.id, 'shape': b.shape, 'size': list(b.size), 'fixed': b.fixed, 'firstFrame': b.first_frame, 'endFrame': b.end_frame}
                   for b in m.bodies],
        'frameCount': m.frame_count,
        'chunks': [{k: c[k] for k in _CHUNK_KEYS} for c in m.chunks],
        'budget': {k: m.budget[k] for k in _BUDGET_KEYS},
    }
    if m.provenance:
        value['provenance'] = dict(m.provenance)
    return _js_value(value)


def _check_keys(d: dict, allowed, what: str, code: str):
    for k in d:
        if k not in allowed:
            _fail(code, f'{what}: unknown field "{re.sub(r"[^ -~]", "?", str(k))[:40]}"')


def _json_no_duplicates(pairs):
    d = {}
    for k, v in pairs:
        if k in d:
            raise ValueError('duplicate key')
        d[k] = v
    return d


def _read_manifest(text, limits: dict) -> PoseCacheManifest:
    if not isinstance(text, str):
        _fail('argument', 'Pose cache manifest: expected text')
    if len(text) > limits['maxManifestBytes']:
        _fail('budget', f'Pose cache manifest is {len(text)} characters; the limit is {limits["maxManifestBytes"]}')
    try:
        value = json.loads(text, object_pairs_hook=_json_no_duplicates)
    except ValueError:
        _fail('manifest', 'Pose cache manifest is not valid JSON (truncated or corrupt?)')
    if not isinstance(value, dict):
        _fail('manifest', 'Pose cache manifest: expected a JSON object')
    if value.get('schema') != POSE_CACHE_SCHEMA:
        _fail('schema', f'Not a pose cache manifest: schema is not {POSE_CACHE_SCHEMA}')
    _check_keys(value, _TOP_KEYS, 'Pose cache manifest', 'manifest')
    if value.get('conventions') != POSE_CACHE_CONVENTIONS:
        _fail('manifest', 'conventions must be exactly metres, seconds, right-handed, y-up, [x, y, z, w] quaternions, little-endian float32')
    cache_id, termination, dt = value.get('cacheId'), value.get('termination'), value.get('dt')
    if not _is_int(cache_id, 0, 0xFFFFFFFF):
        _fail('manifest', 'cacheId must be a caller-assigned unsigned 32-bit integer')
    if termination not in TERMINATIONS:
        _fail('manifest', f'termination must be one of {", ".join(TERMINATIONS)}')
    if not _finite(dt) or dt <= 0 or dt > VALUE_LIMITS['maxDt']:
        _fail('manifest', f'dt must be a number above 0 and at most {VALUE_LIMITS["maxDt"]}')
    if not _is_int(value.get('bodyTableCrc32'), 0, 0xFFFFFFFF):
        _fail('manifest', 'bodyTableCrc32 must be an unsigned 32-bit integer')
    frame_count = value.get('frameCount')
    if not _is_int(frame_count, 1, HARD_LIMITS['maxFrames']):
        _fail('manifest', f'frameCount must be an integer from 1 to {HARD_LIMITS["maxFrames"]}')
    if frame_count > limits['maxFrames']:
        _fail('budget', f'{frame_count} frames exceed the limit of {limits["maxFrames"]}')
    budget = value.get('budget')
    if not isinstance(budget, dict):
        _fail('manifest', 'budget: expected an object')
    _check_keys(budget, _BUDGET_KEYS, 'budget', 'manifest')
    for k, hard in (('maxBodies', 'maxBodies'), ('maxFrames', 'maxFrames'), ('maxBytes', 'maxTotalBytes')):
        if not _is_int(budget.get(k), 1, HARD_LIMITS[hard]):
            _fail('manifest', f'budget.{k} must be an integer from 1 to {HARD_LIMITS[hard]}')
    chunks_in = value.get('chunks')
    if not isinstance(chunks_in, list) or len(chunks_in) < 1:
        _fail('manifest', 'chunks must be a non-empty list')
    if len(chunks_in) > limits['maxChunks']:
        _fail('budget', f'{len(chunks_in)} chunks exceed the limit of {limits["maxChunks"]}')
    bodies = _bodies_from(value.get('bodies'), frame_count, limits, 'manifest')
    if len(bodies) > budget['maxBodies']:
        _fail('manifest', f'{len(bodies)} bodies exceed the declared budget.maxBodies {budget["maxBodies"]}')
    if frame_count > budget['maxFrames']:
        _fail('manifest', f'{frame_count} frames exceed the declared budget.maxFrames {budget["maxFrames"]}')
    if pose_body_table_crc32(dt, bodies, cache_id) != value['bodyTableCrc32']:
        _fail('manifest', 'bodyTableCrc32 does not match cacheId, dt and the body table (edited or corrupt?)')
    frame_bytes, chunks, next_frame, total = pose_frame_bytes(len(bodies)), [], 0, 0
    for i, c in enumerate(chunks_in):
        at = f'chunks[{i}]'
        if not isinstance(c, dict):
            _fail('manifest', f'{at}: expected an object')
        _check_keys(c, _CHUNK_KEYS, at, 'manifest')
        if c.get('index') != i or isinstance(c.get('index'), bool):
            _fail('manifest', f'{at}: index must be {i}')
        if c.get('firstFrame') != next_frame or isinstance(c.get('firstFrame'), bool):
            _fail('manifest', f'{at}: firstFrame must be {next_frame} (chunks are contiguous and in order)')
        if not _is_int(c.get('frameCount'), 1, frame_count - next_frame):
            _fail('manifest', f'{at}: frameCount must be an integer from 1 to {frame_count - next_frame}')
        byte_length = CHUNK_HEADER_BYTES + c['frameCount'] * frame_bytes
        if c.get('byteLength') != byte_length or isinstance(c.get('byteLength'), bool):
            _fail('manifest', f'{at}: byteLength must be {byte_length} (header + {c["frameCount"]} frames of {frame_bytes} bytes)')
        if byte_length > limits['maxChunkBytes']:
            _fail('budget', f'{at}: {byte_length} bytes exceed the chunk limit of {limits["maxChunkBytes"]}')
        total += byte_length
        if total > limits['maxTotalBytes']:
            _fail('budget', f'chunks total more than the limit of {limits["maxTotalBytes"]} bytes')
        chunks.append({'index': i, 'firstFrame': next_frame, 'frameCount': c['frameCount'], 'byteLength': byte_length})
        next_frame += c['frameCount']
    if next_frame != frame_count:
        _fail('manifest', f'chunks hold {next_frame} frames; frameCount is {frame_count}')
    if total > budget['maxBytes']:
        _fail('manifest', f'chunks total {total} bytes, above the declared budget.maxBytes {budget["maxBytes"]}')
    provenance = _provenance_from(value.get('provenance'), 'manifest')
    m = PoseCacheManifest(cache_id, termination, dt, value['bodyTableCrc32'], bodies, frame_count, chunks,
                          {k: budget[k] for k in _BUDGET_KEYS}, provenance)
    # other number spellings, whitespace and key order are refused here: one text per manifest
    if _serialize_manifest(m) != text:
        _fail('manifest', 'Pose cache manifest is not in canonical form (compact JSON, fixed key order, no duplicate keys, no surrounding whitespace)')
    return m


def parse_pose_cache_manifest(text: str, limits: dict | None = None) -> PoseCacheManifest:
    """A manifest alone, parsed and checked (tools that read only the body table or budgets)."""
    return _read_manifest(text, resolve_limits(limits))


# ---- in-memory cache validation -----------------------------------------------------------------

def _normalize_cache(cache: PoseCache, limits: dict) -> PoseCache:
    if not isinstance(cache, PoseCache):
        _fail('argument', 'Pose cache: expected a PoseCache')
    if not _is_int(cache.cache_id, 0, 0xFFFFFFFF):
        _fail('data', 'cacheId must be a caller-assigned unsigned 32-bit integer')
    if not _finite(cache.dt) or cache.dt <= 0 or cache.dt > VALUE_LIMITS['maxDt']:
        _fail('data', f'dt must be a number above 0 and at most {VALUE_LIMITS["maxDt"]}')
    if cache.termination not in TERMINATIONS:
        _fail('data', f'termination must be one of {", ".join(TERMINATIONS)}')
    steps, poses = cache.steps, cache.poses
    if not isinstance(steps, np.ndarray) or steps.dtype != np.uint32 or steps.ndim != 1:
        _fail('argument', 'steps must be a 1-D uint32 array')
    if not isinstance(poses, np.ndarray) or poses.dtype != np.float32:
        _fail('argument', 'poses must be a float32 array (float32 is what the cache stores)')
    frames = len(steps)
    if frames < 1:
        _fail('data', 'a cache needs at least one frame')
    if frames > limits['maxFrames']:
        _fail('budget', f'{frames} frames exceed the limit of {limits["maxFrames"]}')
    bodies = _bodies_from(cache.bodies, frames, limits, 'data')
    if poses.size != frames * len(bodies) * POSE_FLOATS:
        _fail('data', f'poses must hold frames × bodies × 7 = {frames * len(bodies) * POSE_FLOATS} numbers, found {poses.size}')
    frame_bytes = pose_frame_bytes(len(bodies))
    per_chunk = (limits['maxChunkBytes'] - CHUNK_HEADER_BYTES) // frame_bytes
    if per_chunk < 1:
        _fail('budget', f'one frame of {len(bodies)} bodies ({frame_bytes} bytes) does not fit the chunk limit of {limits["maxChunkBytes"]} bytes')
    chunks = -(-frames // per_chunk)
    if chunks > limits['maxChunks']:
        _fail('budget', f'{chunks} chunks exceed the limit of {limits["maxChunks"]}')
    nbytes = frames * frame_bytes + chunks * CHUNK_HEADER_BYTES
    if nbytes > limits['maxTotalBytes']:
        _fail('budget', f'{nbytes} minimum encoded bytes exceed the limit of {limits["maxTotalBytes"]}')
    provenance = _provenance_from(cache.provenance, 'data')
    for f in range(1, frames):
        if steps[f] <= steps[f - 1]:
            _fail('data', f'steps must increase (frame {f}: {int(steps[f])} follows {int(steps[f - 1])})')
    p = poses.reshape(frames, len(bodies), POSE_FLOATS)
    for f in range(frames):
        problem = _frame_problem(p[f], bodies, f)
        if problem:
            _fail('data', problem)
    return PoseCache(cache.cache_id, cache.dt, bodies, steps, p, cache.termination, provenance)


def validate_pose_cache(cache: PoseCache, limits: dict | None = None) -> None:
    """Raise PoseCacheError unless `cache` is complete, consistent and within the limits."""
    _normalize_cache(cache, resolve_limits(limits))


# ---- encode -------------------------------------------------------------------------------------

def encode_pose_cache(cache: PoseCache, frames_per_chunk: int | None = None, limits: dict | None = None, budget: dict | None = None):
    """(manifest text, [chunk bytes]): everything checked first; the chunks are fresh buffers."""
    lim = resolve_limits(limits)
    c = _normalize_cache(cache, lim)
    frames, n = len(c.steps), len(c.bodies)
    frame_bytes = pose_frame_bytes(n)
    most = (lim['maxChunkBytes'] - CHUNK_HEADER_BYTES) // frame_bytes
    if most < 1:
        _fail('budget', f'one frame of {n} bodies ({frame_bytes} bytes) does not fit the chunk limit of {lim["maxChunkBytes"]} bytes')
    per = most if frames_per_chunk is None else frames_per_chunk
    if not _is_int(per, 1, most):
        _fail('argument', f'framesPerChunk must be an integer from 1 to {most}')
    count = -(-frames // per)
    if count > lim['maxChunks']:
        _fail('budget', f'{count} chunks exceed the limit of {lim["maxChunks"]}')
    total = count * CHUNK_HEADER_BYTES + frames * frame_bytes
    if total > lim['maxTotalBytes']:
        _fail('budget', f'{total} bytes exceed the limit of {lim["maxTotalBytes"]}')
    given = {} if budget is None else budget
    if not isinstance(given, dict):
        _fail('argument', 'budget must be a plain object')
    _check_keys(given, _BUDGET_KEYS, 'budget', 'argument')
    b = {'maxBodies': given.get('maxBodies', n), 'maxFrames': given.get('maxFrames', frames), 'maxBytes': given.get('maxBytes', total)}
    if not _is_int(b['maxBodies'], n, HARD_LIMITS['maxBodies']):
        _fail('argument', f'budget.maxBodies must be an integer from {n} (the bodies) to {HARD_LIMITS["maxBodies"]}')
    if not _is_int(b['maxFrames'], frames, HARD_LIMITS['maxFrames']):
        _fail('argument', f'budget.maxFrames must be an integer from {frames} (the frames) to {HARD_LIMITS["maxFrames"]}')
    if not _is_int(b['maxBytes'], total, HARD_LIMITS['maxTotalBytes']):
        _fail('argument', f'budget.maxBytes must be an integer from {total} (the chunk bytes) to {HARD_LIMITS["maxTotalBytes"]}')
    entries = []
    for i, first in enumerate(range(0, frames, per)):
        fc = min(per, frames - first)
        entries.append({'index': i, 'firstFrame': first, 'frameCount': fc, 'byteLength': CHUNK_HEADER_BYTES + fc * frame_bytes})
    table_crc = pose_body_table_crc32(c.dt, c.bodies, c.cache_id)
    manifest = _serialize_manifest(PoseCacheManifest(c.cache_id, c.termination, c.dt, table_crc, c.bodies, frames, entries, b, c.provenance))
    _read_manifest(manifest, lim)  # the writer never emits what its reader refuses
    chunks = []
    for e in entries:
        buf = bytearray(e['byteLength'])
        buf[0:4] = CHUNK_MAGIC
        struct.pack_into('<HHIIIIII', buf, 4, POSE_CACHE_CHUNK_REVISION, CHUNK_HEADER_BYTES, table_crc, e['index'], e['firstFrame'],
                         e['frameCount'], n, e['frameCount'] * frame_bytes)
        head = crc32(buf, 0, 32)
        struct.pack_into('<I', buf, 32, head)
        for j in range(e['frameCount']):
            f, at = e['firstFrame'] + j, CHUNK_HEADER_BYTES + j * frame_bytes
            struct.pack_into('<I', buf, at, int(c.steps[f]))
            buf[at + 4:at + frame_bytes - 4] = np.ascontiguousarray(c.poses[f], dtype='<f4').tobytes()
            struct.pack_into('<I', buf, at + frame_bytes - 4, crc32(buf, at, at + frame_bytes - 4, head))
        chunks.append(bytes(buf))
    return manifest, chunks


# ---- decode and recovery ------------------------------------------------------------------------

def _chunk_header(c: bytes, entry: dict, m: PoseCacheManifest):
    """The chunk's header crc, or the reason it does not match its manifest entry."""
    at = f'chunk {entry["index"]}'
    if len(c) < CHUNK_HEADER_BYTES:
        return f'{at}: ends inside its {CHUNK_HEADER_BYTES}-byte header ({len(c)} bytes)'
    if bytes(c[0:4]) != CHUNK_MAGIC:
        return f'{at}: not a pose cache chunk (bad magic)'
    rev, hsize, table, index, first, fcount, nbodies, payload, head = struct.unpack_from('<HHIIIIIII', c, 4)
    if head != crc32(c, 0, 32):
        return f'{at}: header checksum mismatch (corrupt header)'
    if rev != POSE_CACHE_CHUNK_REVISION:
        return f'{at}: unsupported chunk revision {rev}'
    if hsize != CHUNK_HEADER_BYTES:
        return f'{at}: unexpected header size {hsize}'
    if table != m.body_table_crc32:
        return f'{at}: belongs to a different cache (body table checksum differs from the manifest)'
    if index != entry['index']:
        return f'{at}: header says chunk {index}'
    if first != entry['firstFrame']:
        return f"{at}: first frame {first} differs from the manifest's {entry['firstFrame']}"
    if fcount != entry['frameCount']:
        return f"{at}: {fcount} frames differ from the manifest's {entry['frameCount']}"
    if nbodies != len(m.bodies):
        return f"{at}: {nbodies} bodies differ from the manifest's {len(m.bodies)}"
    want = entry['frameCount'] * pose_frame_bytes(len(m.bodies))
    if payload != want:
        return f'{at}: payload size {payload} differs from {want}'
    return head


def _walk_chunks(m: PoseCacheManifest, chunks):
    """Frames read in order up to the first thing that is not what the manifest promised; memory
    bounded by the bytes supplied."""
    if not isinstance(chunks, (list, tuple)):
        _fail('argument', 'chunks must be a list of bytes')
    if len(chunks) > len(m.chunks):
        _fail('chunk', f'{len(chunks)} chunks given; the manifest lists {len(m.chunks)}')
    for c in chunks:
        if not isinstance(c, (bytes, bytearray, memoryview)):
            _fail('argument', 'every chunk must be bytes')
    n = len(m.bodies)
    frame_bytes = pose_frame_bytes(n)
    heads, problem = [], None
    for i, c in enumerate(chunks):
        h = _chunk_header(c, m.chunks[i], m)
        if isinstance(h, str):
            problem = {'chunk': i, 'frame': m.chunks[i]['firstFrame'], 'code': 'chunk', 'reason': h}
            break
        heads.append(h)
    steps, poses, last = [], [], -1
    for i, head in enumerate(heads):
        c, entry = chunks[i], m.chunks[i]
        available = min(entry['frameCount'], (len(c) - CHUNK_HEADER_BYTES) // frame_bytes)
        broke = None
        for j in range(available):
            at, frame = CHUNK_HEADER_BYTES + j * frame_bytes, len(steps)
            if struct.unpack_from('<I', c, at + frame_bytes - 4)[0] != crc32(c, at, at + frame_bytes - 4, head):
                broke = {'chunk': i, 'frame': frame, 'code': 'data', 'reason': f'frame {frame}: checksum mismatch (corrupt data)'}
                break
            step = struct.unpack_from('<I', c, at)[0]
            if step <= last:
                broke = {'chunk': i, 'frame': frame, 'code': 'data', 'reason': f'steps must increase (frame {frame}: {step} follows {last})'}
                break
            slots = np.frombuffer(bytes(c[at + 4:at + frame_bytes - 4]), dtype='<f4').astype(np.float32).reshape(n, POSE_FLOATS)
            bad = _frame_problem(slots, m.bodies, frame)
            if bad:
                broke = {'chunk': i, 'frame': frame, 'code': 'data', 'reason': bad}
                break
            steps.append(step)
            poses.append(slots)
            last = step
        if broke:
            problem = broke
            break
        if available < entry['frameCount']:
            problem = {'chunk': i, 'frame': len(steps), 'code': 'chunk', 'reason': f'chunk {i}: truncated after {available} of {entry["frameCount"]} frames'}
            break
        extra = len(c) - CHUNK_HEADER_BYTES - entry['frameCount'] * frame_bytes
        if extra > 0:
            problem = {'chunk': i, 'frame': None, 'code': 'chunk', 'reason': f'chunk {i}: {extra} unexpected bytes after its last frame'}
            break
    if problem is None and len(chunks) < len(m.chunks):
        problem = {'chunk': len(chunks), 'frame': m.chunks[len(chunks)]['firstFrame'], 'code': 'chunk',
                   'reason': f'chunk {len(chunks)} of {len(m.chunks)} is missing'}
    s = np.array(steps, dtype=np.uint32)
    p = np.stack(poses) if poses else np.zeros((0, n, POSE_FLOATS), np.float32)
    return s, p, problem


def decode_pose_cache(manifest: str, chunks, limits: dict | None = None) -> PoseCache:
    """A complete cache, or PoseCacheError: no partial result (recover_pose_cache_prefix gives one)."""
    m = _read_manifest(manifest, resolve_limits(limits))
    steps, poses, problem = _walk_chunks(m, chunks)
    if problem:
        _fail(problem['code'], problem['reason'])
    return PoseCache(m.cache_id, m.dt, [PoseCacheBody(b.id, b.shape, list(b.size), b.fixed, b.first_frame, b.end_frame) for b in m.bodies],
                     steps, poses, m.termination, m.provenance)


def recover_pose_cache_prefix(manifest: str, chunks, limits: dict | None = None) -> PoseCacheRecovery:
    """The longest prefix of whole, verified frames and why it stopped. The manifest is the only
    authority on the body table and layout, so an unreadable manifest raises. The recovered cache keeps
    the bodies alive in the prefix, lifetimes clipped to it."""
    m = _read_manifest(manifest, resolve_limits(limits))
    steps, poses, problem = _walk_chunks(m, chunks)
    frames = len(steps)
    if frames == 0:
        return PoseCacheRecovery(None, False, m.frame_count, 0, [b.id for b in m.bodies], problem)
    keep = [i for i, b in enumerate(m.bodies) if b.first_frame < frames]
    if not keep:
        return PoseCacheRecovery(None, False, m.frame_count, frames, [b.id for b in m.bodies], problem)
    bodies = [PoseCacheBody(m.bodies[i].id, m.bodies[i].shape, list(m.bodies[i].size), m.bodies[i].fixed, m.bodies[i].first_frame,
                            min(m.bodies[i].end_frame, frames)) for i in keep]
    cache = PoseCache(m.cache_id, m.dt, bodies, steps, poses[:, keep].copy(), 'recovered' if problem else m.termination, m.provenance)
    return PoseCacheRecovery(cache, problem is None, m.frame_count, frames, [b.id for b in m.bodies if b.first_frame >= frames], problem)


# ---- sampling -----------------------------------------------------------------------------------

def pose_cache_duration(cache: PoseCache) -> float:
    """Seconds from the first frame to the last, by the step stamps."""
    return float(int(cache.steps[-1]) - int(cache.steps[0])) * cache.dt


def sample_pose_cache(cache: PoseCache, time: float, out: np.ndarray, alive: np.ndarray) -> None:
    """The poses at `time` (seconds from the first frame, clamped into the cache) into out (bodies x 7)
    and 1 or 0 per body into alive. At a frame's own time, that frame exactly; between two frames a
    body alive in both moves linearly and turns along the normalized shortest-arc blend (an exact
    cancellation keeps the earlier rotation); a body born or ended in between is absent there."""
    n, steps = len(cache.bodies), cache.steps
    frames = len(steps)
    p = np.asarray(cache.poses, dtype=np.float32).reshape(frames, n, POSE_FLOATS)
    if not math.isfinite(time):
        raise ValueError('sample_pose_cache: time must be finite')
    if out.size != n * POSE_FLOATS or alive.size != n:
        raise ValueError('sample_pose_cache: out must hold bodies x 7 numbers, alive one per body')
    o, a = out.reshape(n, POSE_FLOATS), alive.reshape(n)
    first, dt = int(steps[0]), cache.dt
    at = lambda k: (int(steps[k]) - first) * dt
    t = min(max(time, 0.0), at(frames - 1))
    lo, hi = 0, frames - 1
    while lo < hi:  # the last frame whose time is <= t, in the expression frame times are written in
        mid = (lo + hi + 1) >> 1
        if at(mid) <= t:
            lo = mid
        else:
            hi = mid - 1
    span = 0.0 if lo == frames - 1 else at(lo + 1) - at(lo)
    exact = not (span > 0) or t <= at(lo)
    f = 0.0 if exact else (t - at(lo)) / span
    for i, b in enumerate(cache.bodies):
        in_lo = b.first_frame <= lo < b.end_frame
        live = in_lo if exact else in_lo and b.first_frame <= lo + 1 < b.end_frame
        a[i] = 1 if live else 0
        if not live:
            o[i] = 0
            continue
        x = p[lo, i].astype(np.float64)
        if exact:
            o[i] = x
            continue
        y = p[lo + 1, i].astype(np.float64)
        o[i, :3] = x[:3] + (y[:3] - x[:3]) * f
        s = -1.0 if float(np.dot(x[3:], y[3:])) < 0 else 1.0
        q = x[3:] + (s * y[3:] - x[3:]) * f
        length = math.sqrt(float(np.dot(q, q)))
        o[i, 3:] = q / length if length > 1e-9 else x[3:]
