"""The adjoint of a batched FP32 rollout recorded on the device (avbd_batch_record_start,
avbd_adjoint_create_from_batch): the recording's double-precision replay follows the FP32 rollout,
its gradient equals the oracle's FP64 tape adjoint on the very same recorded structure (read back
and split per world), and agrees with central differences of the replay."""

import numpy as np
import pytest

import avbd_b200
from avbd_b200.adjoint import split
from avbd_b200.scenes import tumbling_world
from oracle import Adjoint as TapeAdjoint

pytestmark = pytest.mark.gpu


def _batch(worlds=6, bodies=16, steps=40, iterations=10, seed=100):
    scenes = [tumbling_world(np.random.default_rng(seed + w), bodies) for w in range(worlds)]
    for s in scenes:
        s.params.iterations = iterations
    b = avbd_b200.BatchSolver3D(worlds, sum(len(s.bodies) for s in scenes), params=scenes[0].params)
    for s in scenes:
        b.add_scene(s)
    return b, scenes


def _params32(sp):
    f = lambda x: float(np.float32(x))
    return {'dt': f(sp.dt), 'gravity': f(sp.gravity), 'alpha': f(sp.alpha), 'gamma': f(sp.gamma), 'beta_lin': f(sp.beta_lin),
            'contact_margin': f(sp.contact_margin), 'iterations': sp.iterations}


def test_recorded_batch_adjoint(cuda_lib):
    steps = 40
    b, scenes = _batch(steps=steps)
    b.record_start(steps)
    b.step(steps)
    b.synchronize()
    st = b.record_status()
    assert st['steps'] == steps and st['problems'] == 0 and st['points'] > 0
    final32 = [b.read_bodies(w) for w in range(len(scenes))]
    adj = avbd_b200.Adjoint.from_batch(b, checkpoint=10)
    info = adj.info()
    assert info['worlds'] == len(scenes) and info['steps'] == steps and info['points'] == st['points']
    p0 = adj.nominal()
    fb = adj.first_body
    # the FP64 replay with the frozen structure follows the FP32 rollout
    _, fin = adj.forward(p0)
    worst_pos = 0.0
    for w, rec in enumerate(final32):
        dyn = rec['mass'] > 0
        worst_pos = max(worst_pos, np.abs(fin[fb[w]:fb[w + 1], :3][dyn] - rec['pos'][dyn]).max())
    print(f'replay vs FP32 rollout after {steps} steps: {worst_pos:.2e} m')
    assert worst_pos < 2e-3
    # target from the replay with perturbed parameters
    rng = np.random.default_rng(3)
    pt = p0.copy()
    pt[0::8] += rng.normal(0, 0.2, adj.bodies)
    pt[5::8] += rng.normal(0, 0.5, adj.bodies)
    _, target = adj.forward(pt)
    adj.set_target(target.reshape(-1))
    loss, g = adj.backward(p0)
    # the FP64 tape adjoint on the same recorded structure, world by world
    rec = adj.read_recording()
    params = _params32(scenes[0].params)
    worst_l = worst_g = 0.0
    for w in range(len(scenes)):
        b0, b1 = int(fb[w]), int(fb[w + 1])
        rw = split(rec, w, params)
        A = TapeAdjoint.from_record(rw, p0[8 * b0:8 * b1])
        A.set_target(target[b0:b1])
        L, gc = A.gradient(p0[8 * b0:8 * b1])
        worst_l = max(worst_l, abs(L - loss[w]) / abs(L))
        dyn = rw['bodies'].reshape(-1, 13)[:, 11] != 0
        G, C = g[8 * b0:8 * b1].reshape(-1, 8)[dyn], gc.reshape(-1, 8)[dyn]
        worst_g = max(worst_g, np.abs(G - C).max() / np.abs(C).max())
    print(f'GPU adjoint vs FP64 tape on the recorded structure: loss rel {worst_l:.2e}, gradient rel {worst_g:.2e}')
    assert worst_l < 1e-9 and worst_g < 1e-5
    # central differences of the replay (h = 1e-6) along a random direction per world
    d = rng.normal(0, 1, p0.shape)
    d[6::8] *= 0.1
    d[7::8] *= 0.05
    dyn_all = np.repeat(rec['bodies'].reshape(-1, 13)[:, 11] != 0, 8)
    d[~dyn_all] = 0.0
    h = 1e-6
    lp, _ = adj.forward(p0 + h * d)
    lm, _ = adj.forward(p0 - h * d)
    fd = (lp - lm) / (2 * h)
    an = np.array([g[8 * fb[w]:8 * fb[w + 1]] @ d[8 * fb[w]:8 * fb[w + 1]] for w in range(len(scenes))])
    rel = np.abs(fd - an) / np.maximum(np.abs(an), 1e-12)
    print('directional derivative rel err per world', rel)
    assert rel.max() < 1e-3
    adj.destroy()
    b.destroy()


def test_recording_refuses_history_and_unsupported_worlds(cuda_lib):
    b, _ = _batch(worlds=2, bodies=8)
    b.step(5)  # contacts now carry warm starts from before any recording
    b.record_start(3)
    b.step(3)
    b.synchronize()
    st = b.record_status()
    if st['problems'] & 2:
        with pytest.raises(avbd_b200.AvbdError):
            avbd_b200.Adjoint.from_batch(b)
    b.destroy()
    # spheres are not differentiated: refused when recording starts
    s = tumbling_world(np.random.default_rng(1), 4)
    s.sphere(0.3, 1.0, 0.5, [0.0, 0.0, 2.0])
    b = avbd_b200.BatchSolver3D(1, len(s.bodies), params=s.params)
    b.add_scene(s)
    with pytest.raises(avbd_b200.AvbdError):
        b.record_start(2)
    b.destroy()
