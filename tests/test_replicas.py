"""The N-GPU replica plumbing (avbd_b200.replicas) with world size 2 over gloo on CPU processes: the
maximum over ranks of the timings, whole-job rates, per-rank seeds and the barrier, as the bench
uses them under torchrun with NCCL."""

import os
import socket

import numpy as np

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from avbd_b200.replicas import Ranks
    R = Ranks.from_env('gloo', timeout_s=60)
    try:
        R.barrier()
        mx = R.max([1.5 + rank, 10.0 - rank, 3.0])
        g = R.all_gather([float(rank), rank + 0.5, -1.0])
        out.put((rank, R.world_size, mx, R.seed(500), R.rate(1000.0, mx[0]), g.tolist()))
        R.barrier()
    finally:
        R.close()


def test_two_ranks_reduce_timings_and_rates():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, world, mx, seed, rate, g in res:
        assert world == 2
        assert mx == [2.5, 10.0, 3.0]          # every rank sees the slowest rank's times
        assert seed == 500 + rank              # replicas draw their own inputs
        assert rate == pytest.approx(2 * 1000.0 / 2.5e-3)  # all ranks' units over the slowest time
        assert g == [[0.0, 0.5, -1.0], [1.0, 1.5, -1.0]]     # every rank's values, in rank order


def test_one_rank_without_environment():
    from avbd_b200.replicas import Ranks
    for k in ('RANK', 'WORLD_SIZE', 'LOCAL_RANK'):
        os.environ.pop(k, None)
    R = Ranks.from_env('gloo')
    assert (R.rank, R.world_size, R.dist) == (0, 1, None)
    assert R.max([4.0, 2.0]) == [4.0, 2.0]
    assert R.all_gather([1.0, 2.0]).tolist() == [[1.0, 2.0]]
    R.barrier()
    R.close()


def _batch_job(count=64, seed=5):
    """A batched job's worlds and their costs, as every rank builds them from one seed."""
    from avbd_b200.replicas import world_cost
    from avbd_b200.scenes import batched_worlds
    scenes = batched_worlds(count, seed=seed)
    costs = []
    for s in scenes:
        pos = np.array([b.pos for b in s.bodies])
        rad = np.array([b.radius for b in s.bodies])
        dyn = np.array([b.mass > 0 for b in s.bodies])
        costs.append(world_cost(pos, rad, dyn, sum(1 for f in s.forces if f.kind != 'ignore')))
    return scenes, np.array(costs)


def _world_result(scene) -> np.ndarray:
    """A stand-in for a world's rollout result (the device calls stubbed): a deterministic function of
    the world's records, a few values per world."""
    pos = np.array([b.pos for b in scene.bodies])
    m = np.array([b.mass for b in scene.bodies])
    return np.array([m.sum(), (pos * m[:, None]).sum(), float(len(scene.bodies))])


def _job_rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    from avbd_b200.replicas import Ranks, partition_worlds
    R = Ranks.from_env('gloo', timeout_s=60)
    try:
        scenes, costs = _batch_job()
        parts = partition_worlds(costs, R.world_size)
        mine = parts[R.rank]
        local = np.stack([_world_result(scenes[i]) for i in mine])
        gathered = R.gather_worlds(mine, local, len(scenes))
        out.put((rank, [p.tolist() for p in parts], gathered.tolist()))
    finally:
        R.close()


def test_batched_job_split_over_two_ranks():
    """One batched job's worlds over two gloo ranks: the partition covers every world exactly once,
    balances Σ(N_w · degree) within one world's cost, is the same on both ranks, and the per-world
    results gathered back in job order equal the one-rank run's, world for world."""
    from avbd_b200.replicas import partition_worlds
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_job_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    scenes, costs = _batch_job()
    single = np.stack([_world_result(s) for s in scenes])
    parts = [np.array(p) for p in res[0][1]]
    assert res[0][1] == res[1][1]  # both ranks split the job alike
    allw = np.sort(np.concatenate(parts))
    assert np.array_equal(allw, np.arange(len(scenes)))  # every world exactly once
    loads = [costs[p].sum() for p in parts]
    assert max(loads) - min(loads) <= costs.max()
    for _, _, gathered in res:
        assert np.array_equal(np.array(gathered), single)
    # more ranks than one: still a cover, still balanced
    for k in (3, 8):
        ps = partition_worlds(costs, k)
        assert np.array_equal(np.sort(np.concatenate(ps)), np.arange(len(costs)))
        ld = [costs[p].sum() for p in ps]
        assert max(ld) - min(ld) <= costs.max()
