"""The N-GPU replica plumbing (avbd_b200.replicas) with world size 2 over gloo on CPU processes: the
maximum over ranks of the timings, whole-job rates, per-rank seeds and the barrier, as the bench
uses them under torchrun with NCCL."""

import os
import socket

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
