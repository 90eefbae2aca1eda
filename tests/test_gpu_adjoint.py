"""The GPU adjoint (avbd_adjoint_*, double precision) against the oracle's FP64 tape adjoint on the
same recorded structures, world by world; the tape adjoint is itself checked against central
differences (tests/test_adjoint_cpu.py)."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200.scenes import tumbling_world
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _recordings(worlds=4, bodies=16, steps=40, seed=0):
    recs, cpu = [], []
    for w in range(worlds):
        s = tumbling_world(np.random.default_rng(seed + w), bodies)
        A = Oracle(s).adjoint(steps)
        recs.append(A.export())
        cpu.append(A)
    return recs, cpu


def test_gpu_adjoint_matches_the_tape_adjoint(cuda_lib):
    recs, cpu = _recordings()
    adj = avbd_b200.Adjoint(recs, checkpoint=10)
    params, targets = [], []
    rng = np.random.default_rng(7)
    for A in cpu:
        p0 = A.nominal()
        pt = p0.copy()
        pt[0::8] += rng.normal(0, 0.2, A.n)
        pt[5::8] += rng.normal(0, 0.5, A.n)
        _, t = A.loss(pt, final=True)
        A.set_target(t)
        params.append(p0)
        targets.append(t.reshape(-1))
    P = np.concatenate(params)
    adj.set_target(np.concatenate(targets))
    loss_f, fin = adj.forward(P)
    loss, g = adj.backward(P)
    assert np.allclose(loss, loss_f, rtol=1e-12)
    o = 0
    worst_g = worst_l = 0.0
    for w, A in enumerate(cpu):
        L, gc = A.gradient(params[w])
        worst_l = max(worst_l, abs(L - loss[w]) / abs(L))
        gw = g[8 * o:8 * (o + A.n)].reshape(-1, 8)
        dyn = recs[w]['bodies'].reshape(-1, 13)[:, 11] != 0  # static bodies have no parameters
        gc = gc.reshape(-1, 8)[dyn]
        gw = gw[dyn]
        worst_g = max(worst_g, np.abs(gw - gc).max() / np.abs(gc).max())
        o += A.n
    print(f'GPU adjoint vs FP64 tape adjoint: loss rel {worst_l:.2e}, gradient rel (to max) {worst_g:.2e}')
    # Both sides are FP64 but sum in different orders (a tape against hand-written cotangents with
    # atomics); contact penalties reach 1e10 against inertia m/dt^2 ~ 1e3, so the 6x6 solves have
    # condition numbers near 1e7 and floored pivots: agreement to 1e-5 of the largest entry.
    assert worst_l < 1e-9 and worst_g < 1e-5
    adj.destroy()
