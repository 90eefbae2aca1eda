"""The pose cache format (src/bake/pose-cache.ts): the codec's byte layout, canonical manifest, checks,
recovery and sampling, on the reference tests' fixture (tests/pose-cache.test.ts:13-30: four bodies,
slot order not id order, one born at frame 2 and one ending before frame 4, frames at steps 0 1 2 4 5 8)."""

import math
import struct

import numpy as np
import pytest

from avbd_b200 import pose_cache as pc

DT, FRAMES, N = 0.25, 6, 4
FB = pc.pose_frame_bytes(N)


def _bodies():
    return [pc.PoseCacheBody(1, 'box', [10, 1, 10], True, 0, 6), pc.PoseCacheBody(20, 'sphere', [1, 1, 1], False, 0, 6),
            pc.PoseCacheBody(9, 'box', [0.5, 0.25, 2], False, 2, 6), pc.PoseCacheBody(5, 'sphere', [2, 2, 2], False, 0, 4)]


def _cache():
    bodies = _bodies()
    poses = np.zeros((FRAMES, N, 7), np.float32)
    for f in range(FRAMES):
        for i, b in enumerate(bodies):
            if b.first_frame <= f < b.end_frame:
                a = 0.3 * f + 0.1 * i
                poses[f, i] = [i + f * 0.5, 10 - f * f * 0.25 + i, -0.125 * f * (i + 1), 0, math.sin(a / 2), 0, math.cos(a / 2)]
    return pc.PoseCache(12345, DT, bodies, np.array([0, 1, 2, 4, 5, 8], np.uint32), poses)


def _raises(fn, code, pattern=None):
    with pytest.raises(pc.PoseCacheError) as e:
        fn()
    assert e.value.code == code, (e.value.code, str(e.value))
    if pattern:
        assert pattern in str(e.value), str(e.value)


def test_crc32_is_the_ieee_crc():
    assert pc.crc32(b'123456789') == 0xCBF43926
    assert pc.crc32(b'') == 0
    assert pc.crc32(bytes([9, 1, 2, 3, 9]), 1, 4) == pc.crc32(bytes([1, 2, 3]))
    data = b'123456789'
    assert pc.crc32(data, 4, len(data), pc.crc32(data, 0, 4)) == 0xCBF43926


def test_numbers_are_spelled_as_javascript_does():
    cases = {0.25: '0.25', 1 / 60: '0.016666666666666666', 1e-7: '1e-7', 1.5e-7: '1.5e-7', 1e21: '1e+21', 1e20: '100000000000000000000',
             1e-6: '0.000001', 10.0: '10', -0.0: '0', 0.1 + 0.2: '0.30000000000000004', 5e-324: '5e-324', 123456.789: '123456.789'}
    for x, want in cases.items():
        assert pc.js_number(x) == want, x


def test_round_trip_bit_for_bit_and_deterministic_encoding():
    c = _cache()
    # float32 corner cases on live slots: negative zero, a subnormal, large and tiny magnitudes
    c.poses[3, 1, :4] = [-0.0, 1e-45, 999999.9375, 1e-30]
    c.poses[1, 0, :3] = [-0.0, -999999.5, 123456.789]
    manifest, chunks = pc.encode_pose_cache(c)
    assert len(chunks) == 1 and len(chunks[0]) == pc.CHUNK_HEADER_BYTES + FRAMES * FB
    back = pc.decode_pose_cache(manifest, chunks)
    assert np.array_equal(back.poses.view(np.uint32), c.poses.view(np.uint32))
    assert np.array_equal(back.steps, c.steps) and [b.id for b in back.bodies] == [1, 20, 9, 5]
    assert back.dt == DT and back.termination == 'complete' and back.provenance is None
    assert np.signbit(back.poses[3, 1, 0]) and 0 < back.poses[3, 1, 1] < 1e-44
    again = pc.encode_pose_cache(back)
    assert again[0] == manifest and again[1] == chunks
    assert pc.pose_cache_duration(back) == 2.0


def test_byte_layout():
    """Magic TAPC, u16 revision 1 and header size 36, u32 body-table CRC, chunk index, first frame,
    frames, bodies, payload bytes, header CRC; then per frame u32 step, f32 slots, chained CRC."""
    one = pc.PoseCache(7, 0.5, [pc.PoseCacheBody(7, 'box', [1, 2, 3], False, 0, 1)], np.array([0x01020304], np.uint32),
                       np.array([1, 2, 3, 0, 0, 0, 1], np.float32))
    manifest, chunks = pc.encode_pose_cache(one)
    c = chunks[0]
    assert c[0:4] == b'TAPC' and list(c[4:8]) == [1, 0, 36, 0]
    assert struct.unpack_from('<I', c, 8)[0] == pc.parse_pose_cache_manifest(manifest).body_table_crc32
    assert struct.unpack_from('<5I', c, 12) == (0, 0, 1, 1, pc.pose_frame_bytes(1))
    assert struct.unpack_from('<I', c, 32)[0] == pc.crc32(c, 0, 32)
    assert list(c[36:40]) == [4, 3, 2, 1] and list(c[40:44]) == [0x00, 0x00, 0x80, 0x3F]
    assert struct.unpack_from('<I', c, len(c) - 4)[0] == pc.crc32(c, 36, len(c) - 4, struct.unpack_from('<I', c, 32)[0])
    assert len(c) == 36 + pc.pose_frame_bytes(1)
    assert manifest.startswith('{"schema":"three-avbd.pose-cache/v0-draft","conventions":{"length":"metre","time":"second",')


def test_any_chunk_size_decodes_to_the_same_cache():
    c = _cache()
    for per in (1, 2, 3, 4, 5, 6, None):
        manifest, chunks = pc.encode_pose_cache(c, frames_per_chunk=per)
        assert len(chunks) == (1 if per is None else -(-FRAMES // per))
        m = pc.parse_pose_cache_manifest(manifest)
        assert sum(e['frameCount'] for e in m.chunks) == FRAMES
        assert all(len(chunks[i]) == e['byteLength'] for i, e in enumerate(m.chunks))
        assert np.array_equal(pc.decode_pose_cache(manifest, chunks).poses, c.poses)
    back = pc.decode_pose_cache(*pc.encode_pose_cache(c, frames_per_chunk=2))
    assert [(b.id, b.first_frame, b.end_frame) for b in back.bodies] == [(1, 0, 6), (20, 0, 6), (9, 2, 6), (5, 0, 4)]


def test_provenance_and_termination_carry():
    c = _cache()
    c.termination, c.provenance = 'cancelled', {'tool': 'unit test', 'gitHead': 'abc123', 'dirty': False, 'steps': 12.5, 'note': None}
    back = pc.decode_pose_cache(*pc.encode_pose_cache(c))
    assert back.termination == 'cancelled' and back.provenance == c.provenance
    c.provenance = {'9bad': 1}
    _raises(lambda: pc.encode_pose_cache(c), 'data', 'provenance')


def test_manifest_is_canonical_and_bound_to_its_body_table():
    manifest, chunks = pc.encode_pose_cache(_cache())
    _raises(lambda: pc.decode_pose_cache(' ' + manifest, chunks), 'manifest', 'canonical')
    _raises(lambda: pc.decode_pose_cache(manifest.replace('"dt":0.25', '"dt":2.5e-1'), chunks), 'manifest', 'canonical')
    _raises(lambda: pc.decode_pose_cache(manifest.replace('"size":[10,1,10]', '"size":[10,1,11]'), chunks), 'manifest', 'bodyTableCrc32')
    _raises(lambda: pc.decode_pose_cache(manifest.replace('three-avbd.pose-cache/v0-draft', 'other'), chunks), 'schema')
    _raises(lambda: pc.decode_pose_cache(manifest[:-5], chunks), 'manifest', 'JSON')
    _raises(lambda: pc.parse_pose_cache_manifest(manifest, {'maxBodies': 3}), 'budget')


def test_corruption_is_found_and_a_prefix_recovered():
    c = _cache()
    manifest, chunks = pc.encode_pose_cache(c, frames_per_chunk=2)
    # a flipped byte in frame 3's poses: its checksum fails, frames 0..2 survive
    bad = bytearray(chunks[1])
    bad[pc.CHUNK_HEADER_BYTES + FB + 10] ^= 1
    _raises(lambda: pc.decode_pose_cache(manifest, [chunks[0], bytes(bad), chunks[2]]), 'data', 'checksum')
    r = pc.recover_pose_cache_prefix(manifest, [chunks[0], bytes(bad), chunks[2]])
    assert not r.complete and r.recovered_frames == 3 and r.declared_frames == 6 and r.problem['frame'] == 3
    assert r.cache.termination == 'recovered' and [b.id for b in r.cache.bodies] == [1, 20, 9, 5]
    assert np.array_equal(r.cache.poses, c.poses[:3])
    # a missing last chunk, a truncated one, a chunk of another cache
    _raises(lambda: pc.decode_pose_cache(manifest, chunks[:2]), 'chunk', 'missing')
    r = pc.recover_pose_cache_prefix(manifest, [chunks[0][:pc.CHUNK_HEADER_BYTES + FB + 3]])
    assert r.recovered_frames == 1 and [b.id for b in r.cache.bodies] == [1, 20, 5] and r.omitted_body_ids == [9]
    other = _cache()
    other.cache_id = 99
    _, foreign = pc.encode_pose_cache(other, frames_per_chunk=2)
    _raises(lambda: pc.decode_pose_cache(manifest, [chunks[0], foreign[1], chunks[2]]), 'chunk', 'different cache')


def test_values_are_checked():
    c = _cache()
    c.poses[1, 3, 6] = 0.5  # not a unit quaternion
    _raises(lambda: pc.encode_pose_cache(c), 'data', 'unit quaternion')
    c = _cache()
    c.poses[0, 2, 0] = 1.0  # body 9 is not alive at frame 0: its slot must be +0
    _raises(lambda: pc.encode_pose_cache(c), 'data', 'outside its lifetime')
    c = _cache()
    c.steps = np.array([0, 1, 1, 4, 5, 8], np.uint32)
    _raises(lambda: pc.encode_pose_cache(c), 'data', 'increase')
    c = _cache()
    c.bodies[1] = pc.PoseCacheBody(20, 'sphere', [1, 2, 1], False, 0, 6)
    _raises(lambda: pc.encode_pose_cache(c), 'data', 'diameter')
    _raises(lambda: pc.encode_pose_cache(_cache(), limits={'maxFrames': 5}), 'budget')
    _raises(lambda: pc.resolve_limits({'maxFrames': 0}), 'argument')


def test_sampling():
    c = pc.decode_pose_cache(*pc.encode_pose_cache(_cache()))
    out, alive = np.zeros((N, 7)), np.zeros(N, np.uint8)
    pc.sample_pose_cache(c, 0.5, out, alive)  # frame 2's own time
    assert list(alive) == [1, 1, 1, 1] and np.array_equal(out, c.poses[2].astype(np.float64))
    pc.sample_pose_cache(c, 0.75, out, alive)  # halfway from frame 2 (0.5 s) to frame 3 (1 s)
    assert np.allclose(out[:, :3], (c.poses[2, :, :3].astype(np.float64) + c.poses[3, :, :3]) / 2)
    assert np.allclose(np.linalg.norm(out[:, 3:], axis=1), 1.0)
    pc.sample_pose_cache(c, 1.1, out, alive)  # between frames 3 and 4: body 5 ends at frame 4
    assert list(alive) == [1, 1, 1, 0] and not out[3].any()
    pc.sample_pose_cache(c, 0.3, out, alive)  # between frames 1 and 2: body 9 is born at frame 2
    assert alive[2] == 0
    pc.sample_pose_cache(c, 99.0, out, alive)  # clamped to the last frame
    assert np.array_equal(out[:3], c.poses[5, :3].astype(np.float64))
