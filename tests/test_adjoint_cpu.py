"""The FP64 CPU adjoint of the step with the contact structure frozen (oracle, test infrastructure):
the replay reproduces the oracle's own GPU-mode rollout, and its tape gradient agrees with central
finite differences (h = 1e-6) of the replay within 1e-3 relative."""

import numpy as np

from avbd_b200.scenes import tumbling_world
from oracle import Oracle


def _problem(bodies=8, steps=30, seed=1):
    s = tumbling_world(np.random.default_rng(seed), bodies)
    o = Oracle(s)
    A = o.adjoint(steps)
    return s, o, A


def test_replay_reproduces_the_oracle_rollout():
    _, o, A = _problem()
    _, fin = A.loss(A.nominal(), final=True)
    b = o.bodies()
    assert np.abs(fin[:, :3] - b[:, 0:3]).max() < 1e-10 and np.abs(fin[:, 3:] - b[:, 3:7]).max() < 1e-10


def test_gradient_matches_central_differences():
    _, _, A = _problem(bodies=8, steps=30, seed=2)
    p0 = A.nominal()
    rng = np.random.default_rng(4)
    pt = p0.copy()
    pt[0::8] += rng.normal(0, 0.2, A.n)
    pt[4::8] += rng.normal(0, 0.5, A.n)
    pt[6::8] *= 1.1
    _, target = A.loss(pt, final=True)
    A.set_target(target)
    L, g = A.gradient(p0)
    assert L > 0
    h = 1e-6
    worst = 0.0
    for j in range(len(p0)):
        if p0[(j // 8) * 8 + 6] <= 0:  # static bodies have no parameters
            continue
        e = np.zeros_like(p0)
        e[j] = h
        fd = (A.loss(p0 + e) - A.loss(p0 - e)) / (2 * h)
        if abs(fd) < 1e-7 and abs(g[j]) < 1e-7:
            continue
        worst = max(worst, abs(fd - g[j]) / max(abs(fd), abs(g[j])))
    print(f'adjoint vs central differences: worst relative error {worst:.2e}')
    assert worst < 1e-3


def test_split_inverts_combine():
    """adjoint.split takes one world back out of a combined (batched) recording."""
    from avbd_b200.adjoint import combine, split
    recs = []
    for w in range(3):
        s = tumbling_world(np.random.default_rng(40 + w), 6 + 3 * w)
        s.params.iterations = 2
        recs.append(Oracle(s).adjoint(12).export())
    c = combine(recs)
    for w, r in enumerate(recs):
        x = split(c, w, r['params'])
        for k in ('bodies', 'step_man', 'step_pt', 'colors', 'ncol'):
            assert np.array_equal(x[k], r[k]), k
        nm, npts = r['manifolds'], r['points']
        for k, n in (('man_bodies', 2 * nm), ('basis', 9 * nm), ('anchors', 6 * npts), ('pt_man', npts), ('pt_prev', npts)):
            assert np.array_equal(x[k][:n], r[k][:n]), k
