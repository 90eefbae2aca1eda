"""One process per GPU for runs on N GPUs (launched by torchrun): the ranks from the environment, a
barrier, the maximum over ranks of per-rank device times, per-rank seeds and whole-job rates.

A single world does not shard (every colour is a Gauss-Seidel pass over the whole world and contacts
cross any cut), so N GPUs run replicas of it. A batched job's worlds are independent: one job's
worlds are split over the ranks (partition_worlds, balanced by each world's bodies times their
expected constraint degree), each rank steps its share, and no collective touches the simulation
data while it steps. The collectives are the barrier, the reduction of the timings (a whole-job
rate divides all ranks' work by the slowest rank's time), and, after a rollout, one reduction that
puts every world's results (losses, gradients, poses) back in the job's world order on every rank
(gather_worlds). NCCL on GPUs; gloo serves the same calls on CPU processes (the tests)."""

from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta

import numpy as np


def world_cost(positions: np.ndarray, radii: np.ndarray, dynamic: np.ndarray, joints: int = 0, reach: float = 1.5) -> float:
    """A world's share of a batched step: its dynamic bodies times their expected constraint degree,
    1 (the body's own inertia row) + bodies within `reach` x the sum of the two bounding radii (the
    neighbours it will likely touch as it settles) + its joints' endpoints, from the world's starting
    records (deterministic: every rank computes the same number)."""
    p = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    r = np.asarray(radii, dtype=np.float64).reshape(-1)
    dyn = np.asarray(dynamic, dtype=bool).reshape(-1)
    if not dyn.any():
        return 0.0
    d2 = ((p[dyn, None, :] - p[None, :, :]) ** 2).sum(axis=2)
    near = d2 <= (reach * (r[dyn, None] + r[None, :])) ** 2
    neighbours = near.sum() - int(dyn.sum())  # not itself
    return float(dyn.sum() + neighbours + 2 * joints)


def partition_worlds(costs, ranks: int) -> list[np.ndarray]:
    """One batched job's worlds over `ranks` ranks, balanced by cost: heaviest world first (ties: the
    lower index) to the rank with the least cost so far (ties: the lower rank). Every world lands on
    exactly one rank; a rank's worlds come back in ascending order. Deterministic."""
    c = np.asarray(costs, dtype=np.float64).reshape(-1)
    order = sorted(range(len(c)), key=lambda i: (-c[i], i))
    load = [0.0] * ranks
    parts: list[list[int]] = [[] for _ in range(ranks)]
    for i in order:
        r = min(range(ranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += c[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


@dataclass
class Ranks:
    rank: int = 0
    world_size: int = 1
    local: int = 0
    device: object = None   # torch.device the reductions run on (None: CPU)
    dist: object = None     # torch.distributed once initialised (None with one rank)

    @classmethod
    def from_env(cls, backend: str = 'nccl', timeout_s: float = 300.0) -> 'Ranks':
        """RANK / WORLD_SIZE / LOCAL_RANK (MASTER_ADDR / MASTER_PORT for the rendezvous) as torchrun
        sets them; one rank without them. With NCCL the rank's GPU is LOCAL_RANK."""
        import torch
        r = cls(int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1')), int(os.environ.get('LOCAL_RANK', '0')))
        if backend == 'nccl':
            torch.cuda.set_device(r.local)
            r.device = torch.device('cuda', r.local)
        if r.world_size > 1:
            import torch.distributed as dist
            kw = {'device_id': r.device} if backend == 'nccl' else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
            r.dist = dist
        return r

    def barrier(self):
        """Every rank here, and this rank's GPU idle."""
        import torch
        if self.dist is not None:
            self.dist.barrier()
        if self.device is not None:
            torch.cuda.synchronize(self.device)

    def max(self, values: list[float]) -> list[float]:
        """Element-wise maximum over ranks (every rank gets it)."""
        import torch
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=self.device)
        if self.dist is not None:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return [float(x) for x in t.tolist()]

    def all_gather(self, values) -> 'np.ndarray':
        """Every rank's `values` (the same shape and dtype on each rank), stacked in rank order:
        shape (world_size, *values.shape), on every rank. One all-gather."""
        import numpy as np
        a = np.ascontiguousarray(values)
        if self.dist is None:
            return a[None].copy()
        import torch
        t = torch.from_numpy(a.copy())
        if self.device is not None:
            t = t.to(self.device)
        out = [torch.empty_like(t) for _ in range(self.world_size)]
        self.dist.all_gather(out, t)
        return torch.stack(out).cpu().numpy()

    def gather_worlds(self, mine: np.ndarray, values, total: int) -> np.ndarray:
        """Every world's values in the job's world order, on every rank: `values` holds this rank's
        worlds (`mine`, a partition_worlds share) one row each; each rank writes its rows into a zero
        array of `total` rows and one all-reduce (sum) combines them (each row has one writer, so the
        sum is exact)."""
        import torch
        v = np.asarray(values, dtype=np.float64)
        out = np.zeros((total,) + v.shape[1:], dtype=np.float64)
        out[np.asarray(mine, dtype=np.int64)] = v
        if self.dist is None:
            return out
        t = torch.from_numpy(out)
        if self.device is not None:
            t = t.to(self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def seed(self, base: int) -> int:
        """A rank's own seed for its replica's synthetic inputs."""
        return base + self.rank

    def rate(self, units_per_rank: float, ms_slowest: float) -> float:
        """Whole-job units per second: every rank's units over the slowest rank's time."""
        return self.world_size * units_per_rank / (ms_slowest / 1000.0)

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
