"""Benchmark of the B200 AVBD step: body-steps/s on the 100k-body drop pile.

A step is one full AVBD step (broadphase, narrowphase, adjacency, colouring, warm starts, 10
iterations of primal + dual, velocities) of one world. The timed region is steps 1..K of the pile's
rollout from its starting lattice (600 steps by default: the whole workload), on a fresh world
after W warm-up steps on another one. Between timed steps a 256 MiB buffer is cleared on the
world's stream so every step starts with a cold L2 (inside the timed region).

Single world: replicas only. With --gpus N (one process per GPU under torchrun) every rank runs its
own 100k world; `value` is all ranks' body-steps over the slowest rank's time.

With --batched-worlds N (4096 by default, 0 to skip) the line also carries `batched`: world-steps/s of
N small worlds (lognormal sizes, median 64 bodies, sigma 0.5, clipped to [16, 512]; stacks or piles on
their own ground) stepped together by the batched entry points, against the same worlds stepped one by
one through the single-world entry points (a sample of them), and the batched step end to end through
host buffers.

--impl reference times the reference's CPU algorithm (the oracle port, GPU-mode rules, all host
threads) on a bounded sample of the same workload: the same generator at 2000 bodies, its whole
rollout.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'three-avbd_b200'))

METRIC = 'body-steps/s @100k boxes'
UNIT = 'body-steps/s'
PILE_BODIES = 100_000
SAMPLE_BODIES = 2_000
PILE_SPACING = 2.7
ROLLOUT = 600
NOMINAL_HBM_GBS = 7700.0  # HGX B200 HBM3e, for context beside the measured copy bandwidth
L2_FLUSH_BYTES = 256 << 20


def workload_config(n_bodies: int, steps: int) -> dict:
    return {
        'workload': f'drop pile: {n_bodies} bodies (70% boxes half-extents U[0.25,0.75], 30% spheres r U[0.2,0.6], density U[0.5,2], '
                    f'friction U[0.3,0.8]) on a jittered 10-layer lattice, random orientations, speed U[0,1]; static ground box; '
                    f'dt 1/60, 10 iterations, g -9.81; timed steps 1..{steps} of the rollout',
        'bodies': n_bodies,
        'iterations': 10,
        'dt': 1 / 60,
        'rollout_steps': ROLLOUT,
        'seed': 1,
        'spatial_sort': 'morton',
        'l2': '256 MiB memset between timed steps, inside the timed region',
    }


def alg_bytes(s) -> float:
    """Algorithmic (minimum) bytes of one topology+solve launch, from the step's own counters:
    B_topo + B_warm + I (B_primal + B_dual) + B_vel with N dynamic bodies, M manifolds, P points,
    A adjacency entries, P2 (dynamic body, point) incidences, J = 0 joints:
      B_topo = 24 M + 16 A + 32 N, B_warm = 144 N, B_primal = 140 N + 92 A + 64 P2,
      B_dual = 144 M + 92 P, B_vel = 88 N."""
    N, M, P, A, P2 = float(s['dynamic_bodies']), float(s['manifolds']), float(s['contacts']), float(s['adjacency']), float(s['incidences'])
    I = 10.0
    return 24 * M + 16 * A + 32 * N + 144 * N + I * (140 * N + 92 * A + 64 * P2 + 144 * M + 92 * P) + 88 * N


def measured_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        return float(json.load(open(path))['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.device}', f'--query-gpu={self.QUERY}', '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ''
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, smax, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for l in getattr(self, 'lines', []):
            f = [x.strip() for x in l.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower() == 'active':
                    reasons.add(name)
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': smax or None, 'reasons': sorted(reasons), 'samples': len(sm)}


def cpu_reference(n_bodies: int, steps: int, threads: int, warmup: int = 0) -> dict:
    """The oracle (the reference's algorithm, GPU-mode rules) on the sampled pile's rollout: `warmup`
    untimed steps on one instance (threads and caches), then steps 1..`steps` of a fresh one."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    from avbd_b200.scenes import drop_pile
    from oracle import Oracle, set_threads
    used = set_threads(threads)
    scene = drop_pile(n_bodies, seed=1)
    if warmup > 0:
        warm = Oracle(scene)
        for _ in range(warmup):
            warm.step_gpu()
        del warm
    o = Oracle(scene)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step_gpu()
    dt = time.perf_counter() - t0
    value = n_bodies * steps / dt
    return {'value': value, 'unit': UNIT, 'cores': used, 'kind': 'port', 'seconds': dt,
            'sample': f'drop pile generator at {n_bodies} bodies (same lattice, distributions and seed), steps 1..{steps} of its rollout, '
                      f'C++ oracle in double (GPU-mode rules), {used} OpenMP threads'}


def cpu_upstream(n_bodies: int, steps: int) -> dict:
    """The oracle in the reference CPU solver's own order (ref/solver.ts:137-223: all-pairs
    broadphase, bodies and forces newest first, one Gauss-Seidel pass) on one thread, steps
    1..`steps` of the sampled pile's rollout."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    from avbd_b200.scenes import drop_pile
    from oracle import Oracle, set_threads
    used = set_threads(1)
    o = Oracle(drop_pile(n_bodies, seed=1))
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    return {'value': n_bodies * steps / dt, 'unit': UNIT, 'cores': used, 'seconds': dt,
            'sample': f'drop pile generator at {n_bodies} bodies, steps 1..{steps}, C++ oracle in double in the reference '
                      'CPU solver\'s order (upstream mode), 1 thread'}


def run_reference(args, rank: int):
    if rank != 0:
        return
    steps = min(args.steps, ROLLOUT)
    warmup = max(args.warmup, 3)
    ref = cpu_reference(SAMPLE_BODIES, steps, os.cpu_count() or 1, warmup)
    line = {
        'metric': METRIC, 'value': ref['value'], 'unit': UNIT, 'n_gpus': args.gpus, 'steps': steps, 'warmup': warmup,
        'ms_per_step': 1000 * ref['seconds'] / steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic', 'impl': 'reference', 'config': workload_config(SAMPLE_BODIES, steps),
        'cpu_baseline': {'value': ref['value'], 'unit': UNIT, 'cores': ref['cores'], 'kind': 'port', 'sample': ref['sample']},
        'e2e': {'value': ref['value'], 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def run_batched(args, R, torch) -> dict:
    """world-steps/s of the batched workload, batched launch against per-world launches."""
    import numpy as np
    import avbd_b200
    from avbd_b200.scenes import batched_worlds

    local, barrier = R.local, R.barrier
    scenes = batched_worlds(args.batched_worlds, seed=R.seed(3))
    n = sum(len(s.bodies) for s in scenes)
    dyn = sum(s.dynamic_count for s in scenes)
    b = avbd_b200.BatchSolver3D(len(scenes), n, 1, params=scenes[0].params, device=local)
    for s in scenes:
        b.add_scene(s)
    tuning = b.tune(2)
    b.step(args.warmup)
    b.synchronize()
    steps = args.batched_steps
    stream = torch.cuda.ExternalStream(b.stream, device=local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f'cuda:{local}')
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            b.step(1)
            flush.zero_()
        e1.record(stream)
    b.synchronize()
    barrier()
    ms, = R.max([e0.elapsed_time(e1)])
    errors = sum(1 for i in range(len(scenes)) if b.read_counters(i)['error'])
    info = b.info()

    # end to end: every step uploads all bodies from pinned host memory and reads them back
    host = torch.empty(n * 160, dtype=torch.uint8).pin_memory()
    host_np = host.numpy().view(avbd_b200.BODY_DTYPE)
    b.read_all_bodies_into(host_np)
    barrier()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            b.write_all_bodies_async(host_np)
            b.step(1)
            b.read_all_bodies_into(host_np, sync=True)
        e1.record(stream)
    b.synchronize()
    barrier()
    te, = R.max([e0.elapsed_time(e1)])
    b.destroy()

    # per-world launches: a sample of the same worlds, each stepped through the single-world API
    sample = scenes[::max(1, len(scenes) // args.plain_sample)][:args.plain_sample]
    worlds = [avbd_b200.CudaSolver3D(s, device=local) for s in sample]
    for w in worlds:
        w.step(args.warmup)
        w.synchronize()
    plain_steps = max(1, min(steps, 30))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(plain_steps):
        for w in worlds:
            w.step(1)
    for w in worlds:
        w.synchronize()
    plain_s = time.perf_counter() - t0
    for w in worlds:
        w.destroy()
    value = R.rate(len(scenes) * steps, ms)
    plain = len(sample) * plain_steps / plain_s
    return {
        'metric': 'world-steps/s', 'value': value, 'ms_per_step': ms / steps, 'steps': steps,
        'body_steps_per_s': R.rate(dyn * steps, ms),
        'per_world_launch': {'value': plain, 'unit': 'world-steps/s', 'sample_worlds': len(sample), 'steps': plain_steps,
                             'how': 'each sampled world stepped through the single-world entry points in turn, wall clock'},
        'speedup_vs_per_world_launch': value / R.world_size / plain,
        'e2e': {'value': R.rate(len(scenes) * steps, te), 'unit': 'world-steps/s',
                'h2d_bytes_per_step': n * 160, 'd2h_bytes_per_step': n * 160},
        'worlds': len(scenes), 'bodies': n, 'dynamic_bodies': dyn, 'world_errors': errors,
        'launch': {'collide_threads': info['collide_threads'], 'collide_blocks': info['collide_blocks'], 'solve_blocks': info['solve_blocks'],
                   'graphs': bool(info['graphs'])},
        'tuning_ms': {f"{c['collide_threads']}x{c['solve_blocks']}": round(c['ms_per_step'], 4) for c in tuning['candidates']},
        'gpu_launches': 2 * steps,
        'config': {'workload': f'{len(scenes)} worlds, bodies per world round(lognormal(median 64, sigma 0.5)) clipped to [16, 512]; '
                               'half stacks of unit cubes, half piles of unit cubes and r 0.5 spheres, each on its own ground box; '
                               f'dt 1/60, 10 iterations; timed steps {args.warmup + 1 + tuning["steps_taken"]}..'
                               f'{args.warmup + tuning["steps_taken"] + steps} after tuning and warm-up',
                   'seed': R.seed(3), 'l2': '256 MiB memset between timed steps, inside the timed region'},
    }


def run_hulls(args, R, torch) -> dict:
    """Config 3: 20k convex hulls falling onto 1000 jointed chains of 50 boxes, 15 iterations."""
    import avbd_b200
    from avbd_b200.scenes import hulls_and_chains

    local, barrier = R.local, R.barrier
    scene = hulls_and_chains(args.hulls, args.chains, 50, seed=R.seed(9))
    w = avbd_b200.CudaSolver3D(scene, device=local, spatial_sort=True)
    w.step(args.warmup)
    w.synchronize()
    steps = args.hull_steps
    w.enable_step_stats(steps)
    stream = torch.cuda.ExternalStream(w.stream, device=local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f'cuda:{local}')
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(steps):
            w.step(1)
            flush.zero_()
        e1.record(stream)
    w.synchronize()
    barrier()
    ms, = R.max([e0.elapsed_time(e1)])
    st = w.read_step_stats()
    c = w.read_counters()
    joints, _ = w.read_joints()
    broken = int((joints['stiffness_lin'] == 0).sum())
    dyn = scene.dynamic_count
    w.destroy()
    return {
        'metric': 'body-steps/s', 'value': R.rate(dyn * steps, ms), 'ms_per_step': ms / steps, 'steps': steps,
        'dynamic_bodies': dyn, 'hull_records': len(scene.hull_offsets), 'joints': len(joints), 'joints_broken': broken,
        'phases_ms_per_step': {'collision': float(st['collision_ms'].mean()), 'topology_solve': float(st['solve_ms'].mean())},
        'last_step': {k: int(st[-1][k]) for k in ('pairs', 'manifolds', 'contacts', 'colors')}, 'error': c['error'], 'overflow': c['overflow'],
        'config': {'workload': f'{args.hulls} hulls (hull of 8-32 points on an ellipsoid, semi-axes U[0.3,1.0]; 512 distinct shapes) falling '
                               f'onto {args.chains} chains of 50 boxes (0.2x0.2x0.5) with ball joints breaking at 1e4 N on pull, hung from static '
                               f'anchors; static ground; dt 1/60, 15 iterations; timed steps {args.warmup + 1}..{args.warmup + steps}',
                   'seed': R.seed(9), 'l2': '256 MiB memset between timed steps, inside the timed region'},
    }


def run_adjoint(args, R, torch) -> dict:
    """Config 5: gradients of a final-pose loss over 1024 worlds of 64 tumbling boxes, 120 steps, 10
    iterations, through the FP64 adjoint (checkpoint every 10 steps) of the recorded FP32 batched
    rollout; the target comes from a seeded FP32 rollout with perturbed parameters. Reported: the FP32
    forward (plain and recording), the adjoint's FP64 replay and reverse sweep, their ratios, and
    central differences (h = 1e-6) of the replay along a random direction on 32 sampled worlds."""
    import numpy as np
    import avbd_b200
    from avbd_b200.scenes import tumbling_world

    W, NB, K = args.adjoint_worlds, 64, args.adjoint_steps
    local, barrier = R.local, R.barrier
    seed = R.seed(500)
    scenes = [tumbling_world(np.random.default_rng(seed * 100003 + w), NB) for w in range(W)]
    n = sum(len(s.bodies) for s in scenes)
    b = avbd_b200.BatchSolver3D(W, n, params=scenes[0].params, device=local)
    for s in scenes:
        b.add_scene(s)
    nominal = np.zeros(n, avbd_b200.BODY_DTYPE)
    b.read_all_bodies_into(nominal)
    nominal['flags'] = 1.0  # written again: no contact history
    dyn = nominal['mass'] > 0
    stream = torch.cuda.ExternalStream(b.stream, device=local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def batch_ms(record: bool) -> float:
        b.write_all_bodies_async(nominal)
        b.synchronize()
        if record:
            b.record_start(K)
        with torch.cuda.stream(stream):
            e0.record(stream)
            b.step(K)
            e1.record(stream)
        b.synchronize()
        return e0.elapsed_time(e1)

    # the target: the FP32 rollout with perturbed parameters
    rng = np.random.default_rng(seed)
    pert = nominal.copy()
    pert['vel'][dyn] += rng.normal(0, 0.2, (int(dyn.sum()), 3)).astype(np.float32)
    pert['ang_vel'][dyn] += rng.normal(0, 0.5, (int(dyn.sum()), 3)).astype(np.float32)
    scale = rng.uniform(0.9, 1.1, int(dyn.sum())).astype(np.float32)
    pert['mass'][dyn] *= scale
    pert['moment'][dyn] *= scale[:, None]
    pert['friction'][dyn] *= rng.uniform(0.9, 1.1, int(dyn.sum())).astype(np.float32)
    b.write_all_bodies_async(pert)
    b.synchronize()
    b.step(K)
    b.synchronize()
    final = np.zeros(n, avbd_b200.BODY_DTYPE)
    b.read_all_bodies_into(final)
    target = np.concatenate([final['pos'], final['rot']], axis=1).astype(np.float64).reshape(-1)
    batch_ms(False)  # warm-up (graphs)
    fwd_plain = batch_ms(False)
    fwd_rec = batch_ms(True)
    rec = b.record_status()
    adj = avbd_b200.Adjoint.from_batch(b, checkpoint=10)
    info = adj.info()
    adj.set_target(target)
    p0 = adj.nominal()
    adj.forward(p0)  # warm-up
    adj.backward(p0)
    dev = torch.cuda.current_stream(local)
    barrier()
    e0.record(dev)
    loss, _ = adj.forward(p0)
    e1.record(dev)
    torch.cuda.synchronize(local)
    replay = e0.elapsed_time(e1)
    e0.record(dev)
    loss_b, grad = adj.backward(p0)
    e1.record(dev)
    torch.cuda.synchronize(local)
    backward = e0.elapsed_time(e1)
    barrier()
    fwd_rec, replay, backward = R.max([fwd_rec, replay, backward])
    # the whole job's per-world losses and gradients on every rank (one all-gather each)
    losses_all = R.all_gather(np.asarray(loss_b, dtype=np.float64))
    grads_all = R.all_gather(np.asarray(grad, dtype=np.float64))
    # central differences of the replay along a random direction, 32 sampled worlds
    fb = adj.first_body.astype(np.int64)
    d = rng.normal(0, 1, p0.shape)
    d[6::8] *= 0.1
    d[7::8] *= 0.05
    d[np.repeat(~dyn, 8)] = 0.0
    # (a world whose loss has a kink within the step along d, a contact switching between sticking and
    # sliding or between touching and separating, shows as central differences at h and 2h that
    # disagree; such worlds are counted apart)
    h = 1e-6
    fd = {}
    for hh in (h, 2 * h):
        lp, _ = adj.forward(p0 + hh * d)
        lm, _ = adj.forward(p0 - hh * d)
        fd[hh] = (lp - lm) / (2 * hh)
    sample = rng.choice(W, size=min(32, W), replace=False)
    rel, rel_all, kinks = [], [], 0
    for w in sample:
        a0, a1 = 8 * fb[w], 8 * fb[w + 1]
        an = float(grad[a0:a1] @ d[a0:a1])
        err = abs(fd[h][w] - an) / max(abs(an), 1e-12)
        rel_all.append(err)
        if abs(fd[h][w] - fd[2 * h][w]) > 1e-3 * max(abs(fd[h][w]), 1e-12):
            kinks += 1
        else:
            rel.append(err)
    adj.destroy()
    b.destroy()
    return {
        'metric': 'adjoint/forward time ratio', 'value': (replay + backward) / fwd_rec, 'unit': 'x', 'higher_is_better': False,
        'forward_fp32_ms': fwd_plain, 'forward_fp32_recording_ms': fwd_rec, 'replay_fp64_ms': replay, 'reverse_fp64_ms': backward,
        'ratio_reverse_to_forward': backward / fwd_rec, 'ratio_replay_plus_reverse_to_forward': (replay + backward) / fwd_rec,
        'loss_mean': float(np.mean(losses_all)), 'gradient_finite': bool(np.isfinite(grads_all).all()),
        'gathered': {'worlds': int(losses_all.size), 'gradient_values': int(grads_all.size)},
        'fd_check': {'worlds': len(sample), 'h': h, 'direction': 'random per world (v0, omega0 unit scale; mass 0.1; friction 0.05)',
                     'smooth_worlds': len(rel), 'max_rel_err_smooth': float(max(rel)) if rel else None,
                     'median_rel_err': float(np.median(rel_all)), 'max_rel_err_all': float(max(rel_all)),
                     'worlds_with_kink_within_2h': kinks},
        'recording': {'manifolds': rec['manifolds'], 'points': rec['points'], 'max_points_per_world_step': info['max_points']},
        'config': {'workload': f'{W} worlds x {NB} boxes (0.8 m, density 1, friction 0.5) tumbling onto a static ground; dt 1/60, '
                               f'10 iterations, {K} steps; FP32 forward, FP64 adjoint with a checkpoint every 10 steps; gradients of the '
                               'squared final-pose distance to a target w.r.t. v0, omega0, mass and friction of every body',
                   'seed': seed, 'target': 'FP32 rollout with v0 + N(0,0.2), omega0 + N(0,0.5), mass and friction x U(0.9,1.1)',
                   'timing': 'CUDA events on the launching stream; the replay and reverse read GBs of snapshots (inputs larger than L2)'},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=ROLLOUT)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='cuda', choices=['cuda', 'reference'])
    ap.add_argument('--bodies', type=int, default=PILE_BODIES)
    ap.add_argument('--spacing', type=float, default=PILE_SPACING,
                    help='lattice spacing of the pile (1.15: bodies start touching, the dense case the profiles capture)')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-graphs', action='store_true', help='launch each kernel directly instead of replaying the step graph')
    ap.add_argument('--batched-worlds', type=int, default=4096, help='worlds of the batched workload (0: skip it)')
    ap.add_argument('--batched-steps', type=int, default=300)
    ap.add_argument('--plain-sample', type=int, default=64, help='worlds stepped one by one for the per-world comparison')
    ap.add_argument('--hull-steps', type=int, default=120, help='timed steps of the hulls-and-chains workload (0: skip it)')
    ap.add_argument('--hulls', type=int, default=20000)
    ap.add_argument('--chains', type=int, default=1000)
    ap.add_argument('--adjoint-worlds', type=int, default=1024, help='worlds of the differentiated batch (0: skip it)')
    ap.add_argument('--adjoint-steps', type=int, default=120)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == 'reference':
        run_reference(args, int(os.environ.get('RANK', '0')))
        return

    import numpy as np
    import torch
    import avbd_b200
    from avbd_b200.replicas import Ranks
    from avbd_b200.scenes import drop_pile

    R = Ranks.from_env('nccl', timeout_s=300)
    rank, world_size, local, barrier = R.rank, R.world_size, R.local, R.barrier

    scene = drop_pile(args.bodies, seed=1, spacing=args.spacing)
    n_dyn = scene.dynamic_count

    def fresh():
        w = avbd_b200.CudaSolver3D(scene, device=local, spatial_sort=True)
        if args.no_graphs:
            w.use_graphs(False)
        return w

    # Warm-up on its own world (module load, first touch), then a fresh world for the timed rollout
    warm = fresh()
    warm.step(args.warmup)
    warm.synchronize()
    warm.destroy()

    w = fresh()
    w.enable_step_stats(args.steps)
    stream = torch.cuda.ExternalStream(w.stream, device=local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f'cuda:{local}')
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                w.step(1)
                flush.zero_()
            end.record(stream)
        w.synchronize()
        barrier()
    ms = start.elapsed_time(end)
    stats = w.read_step_stats()
    counters = w.read_counters()
    graphs = bool(counters['graphs'])
    if counters['error'] or counters['overflow']:
        print(f'warning: counters {counters}', file=sys.stderr)
    w.destroy()

    ms_max, = R.max([ms])
    value = R.rate(n_dyn * args.steps, ms_max)

    # Roofline of the dominant kernel (the cooperative topology+solve launch), over the timed steps
    solve_ms = float(stats['solve_ms'].sum())
    coll_ms = float(stats['collision_ms'].sum())
    bytes_alg = float(sum(alg_bytes(s) for s in stats))
    achieved = bytes_alg / (solve_ms / 1000.0) / 1e9 if solve_ms > 0 else 0.0
    peak, peak_kind = measured_peak()
    traffic = None
    prof = os.path.join(ROOT, 'profiles', 'topology_solve_traffic.json')
    if os.path.exists(prof):
        try:
            tp = json.load(open(prof))
            # dram bytes per algorithmic byte in the captured launch, applied to this run's launches
            traffic = tp['dram_bytes'] / tp['alg_bytes'] * bytes_alg / len(stats)
        except Exception:
            traffic = None

    # End to end through the public API with host buffers: each step uploads the bodies from pinned
    # host memory, steps, and reads the bodies back (World.read's path), then waits for them.
    e2e = None
    if not args.no_e2e:
        w2 = fresh()
        host = torch.empty(w2.body_count * 160, dtype=torch.uint8).pin_memory()
        host_np = host.numpy().view(avbd_b200.BODY_DTYPE)
        w2.read_bodies_into(host_np)
        s2 = torch.cuda.ExternalStream(w2.stream, device=local)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        with torch.cuda.stream(s2):
            e0.record(s2)
            for _ in range(args.steps):
                w2.write_bodies_async(host_np)
                w2.step(1)
                w2.read_bodies_into(host_np, sync=True)
            e1.record(s2)
        w2.synchronize()
        barrier()
        te, = R.max([e0.elapsed_time(e1)])
        nbytes = w2.body_count * 160
        e2e = {'value': R.rate(n_dyn * args.steps, te), 'unit': UNIT, 'h2d_bytes_per_step': nbytes,
               'd2h_bytes_per_step': nbytes}
        w2.destroy()

    hulls = None
    if args.hull_steps > 0:
        hulls = run_hulls(args, R, torch)

    batched = None
    if args.batched_worlds > 0:
        batched = run_batched(args, R, torch)

    adjoint = None
    if args.adjoint_worlds > 0:
        adjoint = run_adjoint(args, R, torch)

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        ref = cpu_reference(SAMPLE_BODIES, ROLLOUT, os.cpu_count() or 1)
        cpu = {k: ref[k] for k in ('value', 'unit', 'cores', 'kind', 'sample')}
        up = cpu_upstream(SAMPLE_BODIES, ROLLOUT)
        cpu['upstream_order_1_thread'] = {k: up[k] for k in ('value', 'unit', 'cores', 'sample')}

    if rank == 0:
        name = avbd_b200.device_info(local)
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world_size, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': ms_max / args.steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
            'data': 'synthetic', 'config': dict(workload_config(args.bodies, args.steps), parallelism=f'replicas x{world_size}', spacing=args.spacing),
            'roofline': {'bound': 'hbm', 'kernel': 'k_topology_solve', 'achieved': achieved, 'peak': peak, 'peak_kind': peak_kind, 'unit': 'GB/s',
                         'frac': achieved / peak, 'traffic': traffic, 'alg_bytes_per_launch': bytes_alg / max(len(stats), 1),
                         'peak_nominal': NOMINAL_HBM_GBS, 'frac_nominal': achieved / NOMINAL_HBM_GBS},
            'phases_ms_per_step': {'collision': coll_ms / max(len(stats), 1), 'topology_solve': solve_ms / max(len(stats), 1)},
            'pile_last_step': dict({k: int(stats[-1][k]) for k in ('pairs', 'manifolds', 'contacts', 'colors', 'dynamic_bodies', 'adjacency', 'incidences')},
                                   alg_bytes=alg_bytes(stats[-1])) if len(stats) else None,
            'gpu_launches': int(stats['launches'].sum()),
            'cuda_graphs': graphs,
            'clocks': clocks.summary(),
            'e2e': e2e,
            'cpu_baseline': cpu,
            'batched': batched,
            'hulls': hulls,
            'adjoint': adjoint,
            'device': name[0] if name else None,
        }
        print(json.dumps(line), flush=True)
    R.close()


if __name__ == '__main__':
    main()
