"""One process per GPU for runs on N GPUs (launched by torchrun): the ranks from the environment, a
barrier, the maximum over ranks of per-rank device times, per-rank seeds and whole-job rates.

A single world does not shard (every colour is a Gauss-Seidel pass over the whole world and contacts
cross any cut), so N GPUs run replicas: each rank steps its own world or its own batch of worlds,
and no collective touches the simulation data while it steps. The collectives are the barrier, the
reduction of the timings (a whole-job rate divides all ranks' work by the slowest rank's time), and,
after a differentiated rollout, one all-gather of every rank's per-world losses and gradients. NCCL
on GPUs; gloo serves the same calls on CPU processes (the tests)."""

from __future__ import annotations

import os
from dataclasses import dataclass
from datetime import timedelta


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
