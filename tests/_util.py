"""Test helpers: the CPU oracle's state as C-ABI records (the reference's seedFrom, gpu/solver.ts:1320-1359)."""

from __future__ import annotations

import math

import numpy as np

import avbd_b200
from avbd_b200 import BODY_DTYPE, CONTACT_DTYPE, INFO_DTYPE, JOINT_DTYPE, MANIFOLD_DTYPE
from avbd_b200 import _abi
from avbd_b200.solver import finite
from oracle import K_IGNORE, K_JOINT, K_MANIFOLD, K_SPRING, NO_COLOR, Oracle, records_from_cuda_bodies, records_from_cuda_contacts

STICK_BIT = _abi.STICK_BIT


def body_records(o: Oracle) -> np.ndarray:
    b = o.bodies()
    out = np.zeros(len(b), dtype=BODY_DTYPE)
    out['pos'] = b[:, 0:3]
    out['friction'] = b[:, 23]
    out['rot'] = b[:, 3:7]
    out['initial_pos'] = b[:, 26:29]
    out['flags'] = 0.0
    out['initial_rot'] = b[:, 29:33]
    out['size'] = b[:, 16:19]
    out['mass'] = b[:, 19]
    out['moment'] = b[:, 20:23]
    out['radius'] = b[:, 24]
    out['inertial_pos'] = b[:, 33:36]
    out['inertial_rot'] = b[:, 36:40]
    out['vel'] = b[:, 7:10]
    out['prev_up_vel'] = b[:, 15]  # up = +z
    out['ang_vel'] = b[:, 10:13]
    out['shape'] = b[:, 25]
    return out


def joint_records(o: Oracle):
    """Live joints and springs in force order (as GpuSolver3D's constructor and seedFrom take them), and ignore pairs."""
    recs, infos, ignores = [], [], []
    for i in range(o.force_count):
        r = o.force(i)
        kind = int(r[0])
        if kind == K_MANIFOLD:
            continue
        if kind == K_IGNORE:
            ignores.append((int(r[1]), int(r[2])))
            continue
        rec = np.zeros(1, dtype=JOINT_DTYPE)[0]
        info = np.zeros(1, dtype=INFO_DTYPE)[0]
        info['a'], info['b'] = int(r[1]), int(r[2])
        if kind == K_JOINT:
            broken = r[26] != 0
            rec['pen_lin'] = r[3:6]
            rec['stiffness_lin'] = 0.0 if broken else finite(r[21])
            rec['pen_ang'] = r[6:9]
            rec['stiffness_ang'] = 0.0 if broken else finite(r[22])
            rec['lam_lin'] = r[9:12]
            rec['fracture'] = -finite(r[23]) if r[24] else finite(r[23])
            rec['lam_ang'] = r[12:15]
            rec['torque_arm'] = r[25]
            rec['c0_lin'][:3] = r[15:18]
            rec['c0_ang'] = r[18:21]
            rec['yield_force'] = finite(r[27])
            rec['break_bend'] = finite(r[28])
            rest = r[29:33] if r[33] else np.array([0, 0, 0, 1.0])
            rec['rest'] = rest
            rec['rest_start'] = r[34:38] if r[38] else rest
            rec['r_a'] = r[39:42]
            rec['r_b'] = r[42:45]
            info['type'] = _abi.T_JOINT
        else:
            rec['stiffness_lin'] = r[45]
            rec['r_a'] = r[39:42]
            rec['spring_rest'] = r[46]
            rec['r_b'] = r[42:45]
            rec['rest'] = [0, 0, 0, 1]
            rec['rest_start'] = [0, 0, 0, 1]
            info['type'] = _abi.T_SPRING
        recs.append(rec)
        infos.append(info)
    return np.array(recs, dtype=JOINT_DTYPE), np.array(infos, dtype=INFO_DTYPE), np.array(ignores, dtype=np.uint32).reshape(-1, 2)


def contact_records(o: Oracle):
    m, c = o.manifolds()
    man = np.zeros(len(m), dtype=MANIFOLD_DTYPE)
    con = np.zeros(len(c), dtype=CONTACT_DTYPE)
    k = 0
    for i, r in enumerate(m):
        cnt = int(r[3])
        man[i]['a'], man[i]['b'], man[i]['first'], man[i]['count'] = int(r[1]), int(r[2]), k, cnt
        man[i]['normal'] = r[4:7]
        man[i]['friction'] = r[7]
        k += cnt
    for j, q in enumerate(c):
        con[j]['r_a'] = q[2:5]
        con[j]['key'] = (int(q[0]) & 0xFFFFFFFF) | (STICK_BIT if q[1] else 0)
        con[j]['r_b'] = q[5:8]
        con[j]['c0_n'] = q[8]
        con[j]['pen'] = q[11:14]
        con[j]['c0_t1'] = q[9]
        con[j]['lam'] = q[14:17]
        con[j]['c0_t2'] = q[10]
    return man, con


def params_struct(p, flags: int = 0):
    s = _abi.Params(dt=p.dt, gravity=p.gravity, alpha=p.alpha, beta_lin=p.beta_lin, beta_ang=p.beta_ang, gamma=p.gamma,
                    contact_margin=p.contact_margin, iterations=p.iterations, flags=flags)
    s.up[0], s.up[1], s.up[2] = 0.0, 0.0, 1.0
    s.wind_speed, s.wind_angle = getattr(p, 'wind_speed', 0.0), getattr(p, 'wind_angle', 0.0)
    s.wind_gust, s.wind_pressure = getattr(p, 'wind_gust', 0.4), getattr(p, 'wind_pressure', 0.0)
    return s


def cuda_from_oracle(o: Oracle, params, flags: int = 0, seed: bool = True, hulls_from=None, **kw) -> avbd_b200.CudaSolver3D:
    """A fresh CUDA world holding the oracle's state (`new GpuSolver3D(device, ref)` + `seedFrom(ref)`);
    `hulls_from`: the scene whose hull buffer the bodies' shape codes name."""
    bodies = body_records(o)
    joints, info, ignores = joint_records(o)
    w = avbd_b200.CudaSolver3D(body_capacity=max(len(bodies), 1), joint_capacity=max(len(joints), 16), **kw)
    w.params = params_struct(params, flags)
    if hulls_from is not None:
        w.add_scene_hulls(hulls_from)
    w.add_bodies(bodies)
    if len(joints):
        w.add_joints(joints, info)
    if len(ignores):
        w.add_ignore_pairs(ignores)
    if seed:
        # seedFrom writes the bodies back keeping their contact history (gpu/solver.ts:1325-1327)
        w.write_bodies(0, bodies, keep_contacts=True)
        man, con = contact_records(o)
        w.seed_contacts(man, con)
    return w


def oracle_sequential_colors(o: Oracle) -> np.ndarray:
    b = o.bodies()
    colors = np.full(len(b), NO_COLOR, dtype=np.uint32)
    nxt = 0
    for i in range(len(b) - 1, -1, -1):
        if b[i, 19] > 0:
            colors[i] = nxt
            nxt += 1
    assert nxt <= 64
    return colors


def pose_diff(cuda_bodies: np.ndarray, oracle_bodies: np.ndarray) -> float:
    d = 0.0
    if len(oracle_bodies):
        d = max(float(np.abs(cuda_bodies['pos'] - oracle_bodies[:, 0:3]).max()), float(np.abs(cuda_bodies['rot'] - oracle_bodies[:, 3:7]).max()))
    return d


def lcg(seed: int):
    """The reference tests' generator: seed = seed * 1103515245 + 12345 (mod 2^32), / 2^32."""
    state = [seed & 0xFFFFFFFF]

    def rand():
        state[0] = (state[0] * 1103515245 + 12345) & 0xFFFFFFFF
        return state[0] / 2 ** 32
    return rand


def qnormalize(q):
    l = math.sqrt((q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) + q[3] * q[3])
    return [q[0] / l, q[1] / l, q[2] / l, q[3] / l]


def _unbig(x):
    """The device's BIG (its stand-in for infinity) back to infinity."""
    x = np.asarray(x, dtype=np.float64)
    return np.where(np.abs(x) >= 1e38, np.sign(x) * np.inf, x)


def oracle_from_cuda(w: avbd_b200.CudaSolver3D, scene, flags: int = 0) -> Oracle:
    """A GPU-mode FP64 oracle holding a CUDA world's state exactly (its f32 values): bodies, colour
    state, joints and last step's contacts. The world must hold `scene`'s bodies in creation order and
    its joints in the scene's force order (CudaSolver3D(scene), no spatial sort)."""
    o = Oracle(scene, flags=flags)
    o.set_bodies(records_from_cuda_bodies(w.read_bodies(), w.read_colors(), o.bodies()))
    joints, _ = w.read_joints()
    k = 0
    for si, f in enumerate(scene.forces):
        if f.kind == 'ignore':
            continue
        j = joints[k]
        k += 1
        if f.kind != 'joint':
            continue
        oi = o.force_of[si]
        r = o.force(oi)
        broken = j['stiffness_lin'] == 0 and j['stiffness_ang'] == 0
        r[3:6] = j['pen_lin']
        r[6:9] = j['pen_ang']
        r[9:12] = j['lam_lin']
        r[12:15] = j['lam_ang']
        r[15:18] = j['c0_lin'][:3]
        r[18:21] = j['c0_ang']
        if broken:
            r[26] = 1.0
        else:
            r[21] = _unbig(j['stiffness_lin'])
            r[22] = _unbig(j['stiffness_ang'])
        r[23] = _unbig(abs(float(j['fracture'])))
        r[24] = 1.0 if j['fracture'] < 0 else 0.0
        r[27] = _unbig(j['yield_force'])
        r[28] = _unbig(j['break_bend'])
        r[29:33] = j['rest']
        r[34:38] = j['rest_start']
        o.set_joint(oi, r)
    o.set_manifolds(*records_from_cuda_contacts(*w.read_contacts()))
    return o


def contact_map(m: np.ndarray, c: np.ndarray) -> dict:
    """(a, b, feature) -> (rA, rB, lambda, penalty) of a CUDA world's contact readback."""
    out = {}
    for rec in m:
        for k in range(int(rec['first']), int(rec['first'] + rec['count'])):
            key = int(c[k]['key']) & ~STICK_BIT & 0xFFFFFFFF
            out[(int(rec['a']), int(rec['b']), key)] = (c[k]['r_a'], c[k]['r_b'], c[k]['lam'].astype(np.float64), c[k]['pen'].astype(np.float64))
    return out


def oracle_contact_map(o: Oracle) -> dict:
    """(a, b, feature) -> (rA, rB, lambda, penalty) of the oracle's manifolds."""
    m, c = o.manifolds()
    out, k = {}, 0
    for rec in m:
        for q in c[k:k + int(rec[3])]:
            out[(int(rec[1]), int(rec[2]), int(q[0]) & ~STICK_BIT & 0xFFFFFFFF)] = (q[2:5], q[5:8], q[14:17], q[11:14])
        k += int(rec[3])
    return out


def pose_rel_diff(cuda_bodies: np.ndarray, oracle_bodies: np.ndarray) -> float:
    """Largest pose difference relative to the pose's magnitude (positions against max(|x|, 1 m);
    rotations are unit quaternions, so absolute)."""
    if not len(oracle_bodies):
        return 0.0
    x = oracle_bodies[:, 0:3]
    dp = np.abs(cuda_bodies['pos'] - x) / np.maximum(np.abs(x), 1.0)
    dq = np.abs(cuda_bodies['rot'] - oracle_bodies[:, 3:7])
    return max(float(dp.max()), float(dq.max()))


# Multiplier parity: a row agrees when |dlambda| <= LAMBDA_REL |lambda| + LAMBDA_FLOOR_M x penalty.
# lambda = penalty x C + lambda_prev, so the floor is the constraint value C agreeing within a
# micron: near-zero rows (friction at rest, a contact at the clamp) carry no relative scale of
# their own, and a penalty of 1e3 to 1e4 turns a C differing in its last f32 bits into a few mN.
LAMBDA_REL = 1e-5
LAMBDA_FLOOR_M = 1e-6


def lambda_parity(gm: dict, om: dict, floor_m: float = LAMBDA_FLOOR_M, rows_of=(0, 1, 2)) -> dict:
    """Every common contact's multiplier rows (`rows_of`: 0 normal, 1 and 2 friction), GPU against
    oracle: the largest |dlambda| as a multiple of its bound (<= 1 passes), the rows compared and how
    many exceed their bound, the largest relative difference of rows above 1e-3 N, and the share of
    those within LAMBDA_REL."""
    worst, worst_rel, rows, within, compared, over = 0.0, 0.0, 0, 0, 0, 0
    sel = list(rows_of)
    for k, (_, _, lam, pen) in gm.items():
        if k not in om:
            continue
        olam, open_ = np.asarray(om[k][2], float)[sel], np.asarray(om[k][3], float)[sel]
        d = np.abs(np.asarray(lam, float)[sel] - olam)
        bound = LAMBDA_REL * np.abs(olam) + floor_m * np.maximum(open_, 1.0)
        worst = max(worst, float((d / bound).max()))
        compared += len(sel)
        over += int((d > bound).sum())
        big = np.abs(olam) > 1e-3
        if big.any():
            r = d[big] / np.abs(olam[big])
            worst_rel = max(worst_rel, float(r.max()))
            rows += int(big.sum())
            within += int((r <= LAMBDA_REL).sum())
    return {'ratio': worst, 'compared': compared, 'over': over, 'worst_rel': worst_rel, 'rows': rows, 'within_rel': within / max(rows, 1)}
