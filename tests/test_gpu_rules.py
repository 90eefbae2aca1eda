"""The GPU-only contact rules on (gpu/solver.ts:174-231: matchNearest, faceBias, startAtRest,
massPenalty; wgsl-collision.ts:20-48, 674-679, 699-762, 839-899; wgsl-solve.ts:294-335) against the
GPU-mode oracle with the same rules: from the oracle's state, with its colouring, one GPU step
against one FP64 step, poses within 1e-5 (the procedure of the coloured pyramid test)."""

import numpy as np
import pytest

from avbd_b200 import _abi
from avbd_b200.scenes import cube_pyramid, drop_pile
from oracle import Oracle
from _util import contact_map, cuda_from_oracle, lambda_parity, oracle_contact_map, pose_diff

pytestmark = pytest.mark.gpu

ALL_RULES = _abi.FLAG_MATCH_NEAREST | _abi.FLAG_FACE_BIAS | _abi.FLAG_START_AT_REST | _abi.FLAG_MASS_PENALTY


@pytest.mark.parametrize('name', ['pyramid', 'pile'])
def test_gpu_only_rules_match_oracle(cuda_lib, name):
    scene = cube_pyramid(20) if name == 'pyramid' else drop_pile(400, seed=5, spacing=1.6, layers=4)
    o = Oracle(scene, flags=ALL_RULES)
    worst = worst_lam = 0.0
    frame = 0
    for at in (30, 90):
        for _ in range(at - frame):
            o.step_gpu()
        frame = at
        o.round_f32()
        w = cuda_from_oracle(o, scene.params, flags=ALL_RULES)
        o.step_gpu()
        frame += 1
        w.set_fixed_colors(o.colors())
        w.step()
        c = w.read_counters()
        assert c['error'] == 0 and c['overflow'] == 0
        d = pose_diff(w.read_bodies(), o.bodies())
        worst = max(worst, d)
        lp = lambda_parity(contact_map(*w.read_contacts()), oracle_contact_map(o))
        worst_lam = max(worst_lam, lp['ratio'])
        w.destroy()
    print(f'{name} with every GPU-only rule: worst pose diff {worst:.3e}, lambda worst |d| / bound {worst_lam:.2f}')
    assert worst < 1e-5
    assert worst_lam <= 1.0
