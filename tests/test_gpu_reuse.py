"""Contact reuse, the reference's production default (reuseContacts, gpu/solver.ts:181, 222;
updateRefs and copyContacts, wgsl-collision.ts:20-44, 706-753) and the substep option
reuseManifolds (wgsl-collision.ts:755-762, gpu/solver.ts:2121-2188), against the GPU-mode FP64 oracle
with the same rules: a CUDA world rolled into contact, its whole state (bodies, colours, contacts,
reference poses, moved steps, manifold generations) loaded into the oracle, then one step of each:
the same pairs, the same reuse decisions (each manifold's generating step, each body's moved step),
the same contact keys and anchors bit for bit, poses within 1e-5 relative."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200 import _abi
from avbd_b200.scenes import drop_pile
from _util import contact_map, oracle_contact_map, oracle_from_cuda, params_struct, pose_rel_diff

pytestmark = pytest.mark.gpu

RULES = _abi.FLAG_MATCH_NEAREST | _abi.FLAG_FACE_BIAS | _abi.FLAG_REUSE_CONTACTS | _abi.FLAG_START_AT_REST | _abi.FLAG_MASS_PENALTY


def _world(scene, flags):
    w = avbd_b200.CudaSolver3D(scene)
    w.params = params_struct(scene.params, flags)
    return w


def _seeded_oracle(w, scene, flags):
    o = oracle_from_cuda(w, scene, flags=flags)
    r = w.read_reuse_state()
    o.set_reuse_state(r['step'], r['refs'], r['moved'], r['generated'])
    return o


def _compare(w, o, where):
    c = w.read_counters()
    assert c['error'] == 0 and c['overflow'] == 0, where
    gm, om = contact_map(*w.read_contacts()), oracle_contact_map(o)
    assert set(gm) == set(om), f'{where}: {len(set(gm) ^ set(om))} contacts differ'
    for k, (ra, rb, _, _) in gm.items():
        assert np.array_equal(ra, om[k][0].astype(np.float32)) and np.array_equal(rb, om[k][1].astype(np.float32)), f'{where}: anchors of {k}'
    rg, ro = w.read_reuse_state(), o.reuse_state()
    assert rg['step'] == ro['step']
    assert np.array_equal(rg['moved'], ro['moved']), f'{where}: {(rg["moved"] != ro["moved"]).sum()} moved steps differ'
    assert np.array_equal(np.sort(rg['generated']), np.sort(ro['generated'])), where
    d = pose_rel_diff(w.read_bodies(), o.bodies())
    print(f'{where}: {len(gm)} contacts, {int((rg["generated"] < rg["step"]).sum())} of {len(rg["generated"])} manifolds kept, pose {d:.2e}')
    assert d < 1e-5, f'{where}: pose {d}'
    return rg


def test_reuse_contacts_matches_oracle(cuda_lib):
    scene = drop_pile(3000, seed=5, spacing=1.3, layers=5)
    w = _world(scene, RULES)
    w.step(120)
    o = _seeded_oracle(w, scene, RULES)
    pairs = {tuple(p) for p in o.pairs().tolist()}
    w.step()
    o.step_gpu()
    assert {tuple(p) for p in w.read_pairs().tolist()} == pairs
    dyn = o.bodies()[:, 19] > 0
    assert np.array_equal(w.read_colors()[dyn], o.colors()[dyn])
    r = _compare(w, o, 'detecting step')
    kept = int((r['generated'] < r['step']).sum())
    assert kept > len(r['generated']) // 10, 'the pile, still settling, keeps a good share of its manifolds'
    assert kept < len(r['generated']), 'and regenerates some'
    w.destroy()


def test_reuse_manifolds_substep_matches_oracle(cuda_lib):
    scene = drop_pile(3000, seed=6, spacing=1.3, layers=5)
    w = _world(scene, RULES)
    w.step(60)
    o = _seeded_oracle(w, scene, RULES)
    before = {(int(m['a']), int(m['b'])) for m in w.read_contacts()[0]}
    w.step(reuse_manifolds=True)
    o.step_gpu(reuse_manifolds=True)
    r = _compare(w, o, 'substep keeping manifolds')
    assert {(int(m['a']), int(m['b'])) for m in w.read_contacts()[0]} == before
    assert np.all(r['generated'] < r['step'])  # nothing generated in the substep
    # the option does not apply after a write that changes the bodies: the step detects as usual
    w.write_bodies(0, w.read_bodies()[:1], keep_contacts=True)
    w.step(reuse_manifolds=True)
    assert np.any(w.read_reuse_state()['generated'] == w.read_counters()['steps'])
    w.destroy()


def test_reuse_in_batched_worlds_matches_single_worlds(cuda_lib):
    """Contact reuse in a batch (per-world reference poses and pair hash): every world bit-identical
    over 40 steps to the same scene stepped alone with a one-block solve and the same rules."""
    from avbd_b200 import BatchSolver3D
    from avbd_b200.scenes import batched_worlds
    scenes = batched_worlds(12, seed=21)
    for s in scenes:
        s.params = scenes[0].params
    n = sum(len(s.bodies) for s in scenes)
    b = BatchSolver3D(len(scenes), n, 1, params=scenes[0].params)
    b.set_params(params_struct(scenes[0].params, RULES))
    for s in scenes:
        b.add_scene(s)
    singles = [_world(s, RULES) for s in scenes]
    for w in singles:
        w.set_solve_blocks(1)
    b.step(40)
    b.synchronize()
    kept = 0
    for i, w in enumerate(singles):
        w.step(40)
        assert np.array_equal(b.read_bodies(i).view(np.uint32), w.read_bodies().view(np.uint32)), scenes[i].name
        r = w.read_reuse_state()
        kept += int((r['generated'] < r['step']).sum())
        w.destroy()
    assert kept > 0
    b.destroy()
