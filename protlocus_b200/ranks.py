"""One process per GPU: the rank plumbing of the batched workloads.

Every DP job, extension request, region, candidate and peptide of the path is
independent, so ranks never exchange data: each rank builds and processes its
own batch (seeded by its rank), and the only collectives are the barrier that
brackets a timed region and the max over ranks of its elapsed time (whole-job
throughput = all ranks' units / the slowest rank's time).  Under torchrun the
environment gives RANK / WORLD_SIZE / LOCAL_RANK; a single process needs none.
"""
from __future__ import annotations

import datetime
import os


class Ranks:
    """Rank, world size and local device of this process, with a barrier and a
    max-over-ranks.  backend "nccl" binds the process to cuda:LOCAL_RANK and
    reduces on the device; "gloo" reduces on the host (CPU tests)."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if backend == "nccl":
            import torch
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def seed(self, base: int) -> int:
        """Workload seed of this rank: base + rank (distinct batches per rank)."""
        return base + self.rank

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """Maximum of x over all ranks (every rank gets it)."""
        if self._dist is None:
            return float(x)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        """Sum of x over all ranks (units processed by the whole job)."""
        if self._dist is None:
            return float(x)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None


def job_rate(units_all_ranks: float, seconds_max_over_ranks: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return units_all_ranks / seconds_max_over_ranks if seconds_max_over_ranks > 0 else 0.0
