"""Benchmark of the B200 AVBD step: body-steps/s on the 100k-body drop pile, in contact.

A step is one full AVBD step (broadphase, narrowphase, adjacency, colouring, warm starts, 10
iterations of primal + dual, velocities) of one world. The pile (100k bodies on a jittered lattice,
70 % boxes and 30 % spheres, falling onto a static ground) is rolled forward untimed for 200 steps,
by when every layer has landed and the contact count has levelled off (about 215k manifolds and
350k points); the last W of those steps are the warm-up, and both step graphs (one per contact
buffer parity) are captured before the clock starts. The timed region is the next K steps (201 ..
200 + K), with a 256 MiB clear of a scratch buffer after each step on the world's stream so that
every step starts with a cold L2.

Single world: replicas only. With --gpus N (one process per GPU under torchrun) every rank runs its
own 100k world; `value` is all ranks' body-steps over the slowest rank's time.

The line also carries, each in a few keys: `phases_ms_per_step` (device-clock phase times of the timed
steps, so that ms_per_step = collision + topology_solve + l2_flush + launch gaps can be checked),
`e2e` (the same window through the public API with the bodies uploaded from and read back to pinned
host memory every step), `cpu_baseline` (the oracle port from the same step-200 state of the same
pile), `drift_vs_fp64` (poses against the FP64 oracle over a short horizon), `hulls` (config 3),
`batched` (config 4) and `adjoint` (config 5).

--impl reference times the reference's algorithm on the host cores (the oracle port, GPU-mode rules,
all host threads) on the same pile and window: it rolls the same generator's pile forward 200 steps
untimed and times the next min(K, 10) steps.
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
PILE_SPACING = 2.7
ROLL = 200              # untimed steps before the timed window: the pile has landed and is in contact
FD_SMOOTH_TOL = 1e-4     # central differences at h and h/4 within this (relative): the loss is smooth there
REF_MAX_STEPS = 10      # timed steps of the CPU runs (a bounded sample of the window)
NOMINAL_HBM_GBS = 7700.0  # HGX B200 HBM3e, for context beside the measured copy bandwidth
L2_FLUSH_BYTES = 256 << 20


def compact(v, digits: int = 4):
    """Floats rounded to `digits` significant digits, recursively: the sub-results at the end of the
    bench line stay short enough to read whole in a log's last lines."""
    if isinstance(v, float):
        return float(f'{v:.{digits}g}')
    if isinstance(v, dict):
        return {k: compact(x, digits) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [compact(x, digits) for x in v]
    return v


def workload_config(n_bodies: int, steps: int, roll: int = ROLL, spacing: float = PILE_SPACING) -> dict:
    return {
        'workload': f'drop pile: {n_bodies} bodies (70% boxes half-extents U[0.25,0.75], 30% spheres r U[0.2,0.6], density U[0.5,2], '
                    f'friction U[0.3,0.8]) on a jittered 10-layer lattice (spacing {spacing}), random orientations, speed U[0,1]; '
                    f'static ground box; dt 1/60, 10 iterations, g -9.81; rolled {roll} steps untimed, timed steps {roll + 1}..{roll + steps}',
        'bodies': n_bodies, 'iterations': 10, 'seed': 1, 'window': [roll + 1, roll + steps],
        'l2': '256 MiB clear between timed steps, inside the timed region',
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
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while it is open."""

    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.device}', f'--query-gpu={self.QUERY}', '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def stop(self):
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
        for l in self.lines:
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


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle
    return oracle


def cpu_reference(n_bodies: int, roll: int, steps: int, threads: int, spacing: float = PILE_SPACING) -> dict:
    """The reference's algorithm (the oracle port, GPU-mode rules, double) on `threads` host threads:
    the pile rolled `roll` steps untimed, then steps roll+1 .. roll+steps timed."""
    from avbd_b200.scenes import drop_pile
    orc = _oracle()
    used = orc.set_threads(threads)
    o = orc.Oracle(drop_pile(n_bodies, seed=1, spacing=spacing))
    for _ in range(roll):
        o.step_gpu()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step_gpu()
    dt = time.perf_counter() - t0
    return {'value': n_bodies * steps / dt, 'unit': UNIT, 'cores': used, 'kind': 'port', 'seconds': dt,
            'sample': f'the same pile ({n_bodies} bodies, same generator and seed) rolled {roll} steps on the host, steps {roll + 1}..{roll + steps} timed; '
                      f'C++ oracle in double (GPU-mode rules), {used} OpenMP threads'}


def cpu_upstream_pyramid(steps: int = 60, fp32: bool = False) -> dict:
    """Config 1 (the 210-cube pyramid, the reference's CPU-runnable case) in the reference CPU solver's
    own order (ref/solver.ts:137-223: all-pairs broadphase, bodies and forces newest first, one
    Gauss-Seidel pass), the oracle in double (or in float) on one thread, steps 1..`steps`."""
    from avbd_b200.scenes import cube_pyramid
    orc = _oracle()
    used = orc.set_threads(1)
    o = orc.Oracle(cube_pyramid(20), fp32=fp32)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    kind = 'float' if fp32 else 'double'
    return {'value': 210 * steps / dt, 'unit': UNIT, 'cores': used, 'ms_per_step': 1000 * dt / steps,
            'sample': f'210-cube pyramid, steps 1..{steps}, the reference CPU solver\'s order, oracle in {kind}, 1 thread'}


def run_reference(args, rank: int):
    if rank != 0:
        return
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    ref = cpu_reference(args.bodies, args.roll, steps, os.cpu_count() or 1, args.spacing)
    line = {
        'metric': METRIC, 'value': ref['value'], 'unit': UNIT, 'n_gpus': args.gpus, 'steps': steps, 'warmup': args.warmup,
        'ms_per_step': 1000 * ref['seconds'] / steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic', 'impl': 'reference', 'config': workload_config(args.bodies, steps, args.roll, args.spacing),
        'cpu_baseline': {'value': ref['value'], 'unit': UNIT, 'cores': ref['cores'], 'kind': 'port', 'sample': ref['sample']},
        'e2e': {'value': ref['value'], 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def pile_cpu_and_drift(scene, local: int, roll: int, steps: int) -> tuple[dict, dict]:
    """The CPU baseline and the short-horizon drift at the timed window: a world holding the pile in
    creation order is rolled to step `roll` (the same workload at the same step as the timed world; its
    other body order gives other colourings, so not the same bits), its bodies, colours and contacts are
    loaded into the FP64 oracle, then both advance `steps` steps; the oracle's steps are timed on all
    host threads, and the largest pose differences are taken after each step."""
    import numpy as np
    import avbd_b200
    orc = _oracle()
    w = avbd_b200.CudaSolver3D(scene, device=local)
    w.step(roll)
    w.synchronize()
    used = orc.set_threads(os.cpu_count() or 1)
    o = orc.Oracle(scene)
    m, c = w.read_contacts()
    o.load_cuda_state(w.read_bodies(), w.read_colors(), m, c)
    drift, seconds = [], 0.0
    for _ in range(steps):
        w.step(1)
        t0 = time.perf_counter()
        o.step_gpu()
        seconds += time.perf_counter() - t0
        g, ob = w.read_bodies(), o.bodies()
        drift.append((float(np.abs(g['pos'] - ob[:, 0:3]).max()), float(np.abs(g['rot'] - ob[:, 3:7]).max())))
    w.destroy()
    n = len(scene.bodies) - 1
    cpu = {'value': n * steps / seconds, 'unit': UNIT, 'cores': used, 'kind': 'port',
           'sample': f'the same pile at step {roll} (read back from a GPU world and loaded into the oracle), steps '
                     f'{roll + 1}..{roll + steps}; C++ oracle in double (GPU-mode rules), {used} OpenMP threads'}
    pile = {'start': roll, 'steps': steps, 'max_abs_pos_m': [round(d[0], 9) for d in drift], 'max_abs_rot': [round(d[1], 9) for d in drift]}
    return cpu, pile


def pyramid_drift(local: int, steps: int = 60) -> dict:
    """Config 1 (the 210-cube pyramid) from its scene state: the CUDA step against the FP64 oracle's
    GPU-mode step (its own Jones-Plassmann colouring), largest pose differences at a few steps."""
    import numpy as np
    import avbd_b200
    from avbd_b200.scenes import cube_pyramid
    orc = _oracle()
    scene = cube_pyramid(20)
    o = orc.Oracle(scene)
    o.round_f32()
    w = avbd_b200.CudaSolver3D(scene, device=local)
    out = {}
    for k in range(1, steps + 1):
        w.step(1)
        o.step_gpu()
        if k in (1, 10, 30, steps):
            g, ob = w.read_bodies(), o.bodies()
            out[str(k)] = [float(np.abs(g['pos'] - ob[:, 0:3]).max()), float(np.abs(g['rot'] - ob[:, 3:7]).max())]
    w.destroy()
    return {'steps_pos_rot': out}


def job_share(R, scenes):
    """This rank's worlds of one batched job (all ranks build the same job from one seed): the
    partition by Σ(N_w · degree), and the indices of this rank's share."""
    import numpy as np
    from avbd_b200.replicas import partition_worlds, world_cost
    if R.world_size == 1:
        return np.arange(len(scenes))
    costs = [world_cost(np.array([b.pos for b in s.bodies]), np.array([b.radius for b in s.bodies]), np.array([b.mass > 0 for b in s.bodies]),
                        sum(1 for f in s.forces if f.kind != 'ignore')) for s in scenes]
    return partition_worlds(costs, R.world_size)[R.rank]


def run_batched(args, R, torch) -> dict:
    """World-steps/s of the batched workload (config 4), the batched launch against per-world launches.
    On N ranks one job of N x the worlds is split over them (weak scaling)."""
    import avbd_b200
    from avbd_b200.scenes import batched_worlds

    local, barrier = R.local, R.barrier
    job = batched_worlds(args.batched_worlds * R.world_size, seed=3)
    mine = job_share(R, job)
    scenes = [job[i] for i in mine]
    n = sum(len(s.bodies) for s in scenes)
    dyn = sum(s.dynamic_count for s in scenes)
    b = avbd_b200.BatchSolver3D(len(scenes), n, 1, params=scenes[0].params, device=local)
    for s in scenes:
        b.add_scene(s)
    # the worlds land and settle first (untimed), so the tuner times launch shapes on the contact
    # structure the timed window has, not on the first steps' free fall
    if args.batched_settle > 0:
        b.step(args.batched_settle)
    b.synchronize()
    tuning = b.tune(2)
    b.step(args.warmup)
    b.synchronize()
    steps = args.batched_steps
    stream = torch.cuda.ExternalStream(b.stream, device=local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f'cuda:{local}')
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        flush.zero_()
    b.synchronize()
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
    value = len(job) * steps / (ms / 1000.0)
    plain = len(sample) * plain_steps / plain_s
    return {
        'value': value, 'unit': 'world-steps/s', 'ms_per_step': ms / steps, 'steps': steps,
        'speedup_vs_per_world_launch': value / R.world_size / plain,
        'per_world_launch': plain, 'per_world_sample': len(sample),
        'e2e': len(job) * steps / (te / 1000.0), 'h2d_d2h_bytes_per_step': n * 160,
        'worlds': len(job), 'worlds_this_rank': len(scenes), 'dynamic_bodies': dyn, 'world_errors': errors,
        'launch': f"{tuning['collide_threads']}x{tuning['solve_blocks']}x{tuning['rows_per_lane']}x{tuning['world_threads']}",
        'tuning': {'candidates': len(tuning['candidates']), 'best_ms': min(c['ms_per_step'] for c in tuning['candidates']),
                   'worst_ms': max(c['ms_per_step'] for c in tuning['candidates'])},
        'window': [args.batched_settle + tuning['steps_taken'] + args.warmup + 1, args.batched_settle + tuning['steps_taken'] + args.warmup + steps],
        'seed': 3,
    }


def run_hulls(args, R, torch) -> dict:
    """Config 3: 20k convex hulls falling onto 1000 jointed chains of 50 boxes, 15 iterations."""
    import avbd_b200
    from avbd_b200.scenes import hulls_and_chains

    local, barrier = R.local, R.barrier
    scene = hulls_and_chains(args.hulls, args.chains, 50, seed=R.seed(9))
    w = avbd_b200.CudaSolver3D(scene, device=local, spatial_sort=True)
    steps = args.hull_steps
    w.enable_step_stats(steps)
    w.step(args.hull_roll)
    w.synchronize()
    stream = torch.cuda.ExternalStream(w.stream, device=local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f'cuda:{local}')
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        flush.zero_()
    w.synchronize()
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
        'value': R.rate(dyn * steps, ms), 'unit': UNIT, 'ms_per_step': ms / steps, 'steps': steps,
        'window': [args.hull_roll + 1, args.hull_roll + steps], 'dynamic_bodies': dyn, 'joints_broken': broken,
        'phases_ms_per_step': {'collision': round(float(st['collision_ms'].mean()), 4), 'topology_solve': round(float(st['solve_ms'].mean()), 4)},
        'mean_manifolds': int(st['manifolds'].mean()), 'mean_contacts': int(st['contacts'].mean()), 'error': c['error'], 'overflow': c['overflow'],
        'seed': R.seed(9),
    }


def run_adjoint(args, R, torch) -> dict:
    """Config 5: gradients of a final-pose loss over 1024 worlds of 64 tumbling boxes, 120 steps, 10
    iterations, through the FP64 adjoint (checkpoint every 10 steps) of the recorded FP32 batched
    rollout; the target comes from a seeded FP32 rollout with perturbed parameters. Reported: the FP32
    forward (plain and recording), the adjoint's FP64 replay and reverse sweep, their ratios, and
    central differences (h = 1e-6) of the replay along a random direction on 32 sampled worlds, every
    sampled world counted (the replay keeps the recorded contact structure, so the +h and -h rollouts
    differ only where a friction cone or a penalty clamp switches branch, which the difference quotient
    straddles)."""
    import numpy as np
    import avbd_b200
    from avbd_b200.scenes import tumbling_world

    NB, K = 64, args.adjoint_steps
    local, barrier = R.local, R.barrier
    seed = 500
    # one job of world_size x the worlds, split over the ranks
    job = [tumbling_world(np.random.default_rng(seed * 100003 + w), NB) for w in range(args.adjoint_worlds * R.world_size)]
    mine = job_share(R, job)
    scenes = [job[i] for i in mine]
    W = len(scenes)
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
    rng = np.random.default_rng(seed + R.rank)
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
    # the whole job's per-world losses and gradients in job order on every rank (one reduction each)
    losses_all = R.gather_worlds(mine, np.asarray(loss_b, dtype=np.float64), len(job))
    grads_all = R.gather_worlds(mine, np.asarray(grad, dtype=np.float64).reshape(W, -1), len(job))
    # central differences of the replay along a random direction, 32 sampled worlds
    fb = adj.first_body.astype(np.int64)
    d = rng.normal(0, 1, p0.shape)
    d[6::8] *= 0.1
    d[7::8] *= 0.05
    d[np.repeat(~dyn, 8)] = 0.0
    h = 1e-6
    lp, _ = adj.forward(p0 + h * d)
    lm, _ = adj.forward(p0 - h * d)
    fd = (lp - lm) / (2 * h)
    # the same differences at h / 4: where the loss is smooth over [-h, h] the two agree to O(h^2);
    # where a friction-cone or clamp switch lies inside they do not. The rule looks at the replay
    # alone, never at the adjoint, so the smooth set is fixed before the comparison.
    lp4, _ = adj.forward(p0 + 0.25 * h * d)
    lm4, _ = adj.forward(p0 - 0.25 * h * d)
    fd4 = (lp4 - lm4) / (0.5 * h)
    sample = rng.choice(W, size=min(32, W), replace=False)
    rel_all, smooth = [], []
    for w in sample:
        a0, a1 = 8 * fb[w], 8 * fb[w + 1]
        an = float(grad[a0:a1] @ d[a0:a1])
        rel_all.append(abs(fd[w] - an) / max(abs(an), 1e-12))
        smooth.append(abs(fd[w] - fd4[w]) <= FD_SMOOTH_TOL * max(abs(fd[w]), abs(fd4[w]), 1e-12))
    rel_smooth = [e for e, s in zip(rel_all, smooth) if s]
    adj.destroy()
    b.destroy()
    return {
        'value': (replay + backward) / fwd_rec, 'unit': 'x (adjoint / forward time)', 'higher_is_better': False,
        'forward_fp32_ms': round(fwd_plain, 3), 'forward_fp32_recording_ms': round(fwd_rec, 3), 'replay_fp64_ms': round(replay, 3),
        'reverse_fp64_ms': round(backward, 3), 'reverse_over_forward': backward / fwd_rec,
        'loss_mean': float(np.mean(losses_all)), 'gradient_finite': bool(np.isfinite(grads_all).all()), 'gathered_worlds': int(losses_all.size),
        'fd_check': {'worlds': len(sample), 'h': h, 'max_rel_err': float(max(rel_all)), 'median_rel_err': float(np.median(rel_all)),
                     'worlds_within_1e-3': int(sum(1 for e in rel_all if e <= 1e-3)),
                     'smooth_rule': f'|fd(h) - fd(h/4)| <= {FD_SMOOTH_TOL} relative', 'smooth_worlds': len(rel_smooth),
                     'smooth_max_rel_err': float(max(rel_smooth)) if rel_smooth else None,
                     'smooth_median_rel_err': float(np.median(rel_smooth)) if rel_smooth else None},
        'recording': {'manifolds': rec['manifolds'], 'points': rec['points']}, 'seed': seed,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=100)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='cuda', choices=['cuda', 'reference'])
    ap.add_argument('--bodies', type=int, default=PILE_BODIES)
    ap.add_argument('--roll', type=int, default=ROLL, help='untimed steps before the timed window of the pile')
    ap.add_argument('--spacing', type=float, default=PILE_SPACING, help="the pile's lattice spacing (1.15: in contact from the first step)")
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-graphs', action='store_true', help='launch each kernel directly instead of replaying the step graph')
    ap.add_argument('--batched-worlds', type=int, default=4096, help='worlds of the batched workload (0: skip it)')
    ap.add_argument('--batched-steps', type=int, default=300)
    ap.add_argument('--batched-settle', type=int, default=60, help='untimed steps of the batched worlds before the tuner')
    ap.add_argument('--plain-sample', type=int, default=64, help='worlds stepped one by one for the per-world comparison')
    ap.add_argument('--hull-steps', type=int, default=120, help='timed steps of the hulls-and-chains workload (0: skip it)')
    ap.add_argument('--hull-roll', type=int, default=60, help='untimed steps before the hulls-and-chains window (the hulls reach the chains)')
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

    # The timed world: rolled untimed to step ROLL (its last `warmup` steps are the warm-up). Step
    # statistics are on from the start, so both step graphs are captured and instantiated in the roll.
    w = avbd_b200.CudaSolver3D(scene, device=local, spatial_sort=True)
    if args.no_graphs:
        w.use_graphs(False)
    w.enable_step_stats(args.steps)
    w.step(max(args.roll - args.warmup, 0))
    w.step(args.warmup)
    w.synchronize()
    cap0 = w.read_counters()['pair_capacity']
    stream = torch.cuda.ExternalStream(w.stream, device=local)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=f'cuda:{local}')
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the clear alone, K times (its share of ms_per_step), after one untimed clear that loads its kernel
    with torch.cuda.stream(stream):
        flush.zero_()
    w.synchronize()
    with torch.cuda.stream(stream):
        start.record(stream)
        for _ in range(args.steps):
            flush.zero_()
        end.record(stream)
    w.synchronize()
    flush_ms = start.elapsed_time(end) / args.steps
    clocks = ClockSampler(local).start()
    time.sleep(0.5)
    barrier()
    with torch.cuda.stream(stream):
        start.record(stream)
        h0 = time.perf_counter()
        for _ in range(args.steps):
            w.step(1)
            flush.zero_()
        h1 = time.perf_counter()
        end.record(stream)
    w.synchronize()
    barrier()
    clocks.stop()
    ms = start.elapsed_time(end)
    stats = w.read_step_stats()
    counters = w.read_counters()
    graphs = bool(counters['graphs'])
    if counters['error'] or counters['overflow']:
        print(f'warning: counters {counters}', file=sys.stderr)

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
    K = max(len(stats), 1)
    phases = {'collision': coll_ms / K, 'topology_solve': solve_ms / K, 'l2_flush': flush_ms}
    phases['launch_gaps'] = ms_max / args.steps - sum(phases.values())
    phases = {k: round(v, 4) for k, v in phases.items()}

    # End to end through the public API with host buffers, on the same world's next K steps: each step
    # uploads the bodies from pinned host memory, steps, and reads the bodies back (World.read's path).
    e2e = None
    if not args.no_e2e:
        host = torch.empty(w.body_count * 160, dtype=torch.uint8).pin_memory()
        host_np = host.numpy().view(avbd_b200.BODY_DTYPE)
        w.read_bodies_into(host_np)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                w.write_bodies_async(host_np)
                w.step(1)
                w.read_bodies_into(host_np, sync=True)
            e1.record(stream)
        w.synchronize()
        barrier()
        te, = R.max([e0.elapsed_time(e1)])
        nbytes = w.body_count * 160
        e2e = {'value': R.rate(n_dyn * args.steps, te), 'unit': UNIT, 'h2d_bytes_per_step': nbytes, 'd2h_bytes_per_step': nbytes,
               'window': [args.roll + args.steps + 1, args.roll + 2 * args.steps]}
    cap1 = w.read_counters()['pair_capacity']
    last = stats[-1] if len(stats) else None
    w.destroy()

    cpu, drift = None, None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu, pile_drift = pile_cpu_and_drift(scene, local, args.roll, REF_MAX_STEPS)
        cpu['upstream_order_pyramid_1_thread'] = cpu_upstream_pyramid()
        cpu['upstream_order_pyramid_1_thread_f32'] = cpu_upstream_pyramid(fp32=True)
        drift = {'pile': pile_drift, 'pyramid_210': pyramid_drift(local)}

    hulls = run_hulls(args, R, torch) if args.hull_steps > 0 else None
    batched = run_batched(args, R, torch) if args.batched_worlds > 0 else None
    adjoint = run_adjoint(args, R, torch) if args.adjoint_worlds > 0 else None

    if rank == 0:
        name = avbd_b200.device_info(local)
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world_size, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': ms_max / args.steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
            'data': 'synthetic', 'config': dict(workload_config(args.bodies, args.steps, max(args.roll, args.warmup), args.spacing), parallelism=f'replicas x{world_size}'),
            'roofline': {'bound': 'hbm', 'kernel': 'k_topology_solve', 'achieved': achieved, 'peak': peak, 'peak_kind': peak_kind, 'unit': 'GB/s',
                         'frac': achieved / peak, 'traffic': traffic, 'alg_bytes_per_launch': bytes_alg / K,
                         'frac_of_nominal_7700': achieved / NOMINAL_HBM_GBS},
            'phases_ms_per_step': phases,
            'host_enqueue_ms_per_step': round(1000 * (h1 - h0) / args.steps, 4),
            'window_counters': {k: int(np.mean(stats[k])) for k in ('pairs', 'manifolds', 'contacts', 'colors', 'dynamic_bodies')} if last is not None else None,
            'pair_capacity_grew_in_window': bool(cap1 != cap0),
            'gpu_launches': int(stats['launches'].sum()),
            'cuda_graphs': graphs,
            'clocks': clocks.summary(),
            'e2e': e2e,
            'cpu_baseline': compact(cpu),
            'drift_vs_fp64': compact(drift, 3),
            'device': name[0] if name else None,
            # the other workloads last and compact, so that a log's tail holds them whole
            'hulls': compact(hulls),
            'batched': compact(batched),
            'adjoint': compact(adjoint),
        }
        print(json.dumps(line), flush=True)
    R.close()


if __name__ == '__main__':
    main()
