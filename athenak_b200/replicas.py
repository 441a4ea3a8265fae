"""One process per GPU, each running the whole workload as an independent replica.

The drag step of a pack does not shard here (each rank's MeshBlocks stand alone; there is no
data-path collective), so the process group is plumbing only: a barrier on both sides of the
timed region, the largest time over the ranks, and the whole-job throughput as the units all
ranks processed over that time.  NCCL on GPUs; gloo serves the same calls on CPU (tests).
A rank that is gone makes the others' next barrier or reduction end with an error after the
group's timeout instead of waiting for ever.
"""
from __future__ import annotations

import os
from datetime import timedelta


class Replicas:
    def __init__(self, world: int | None = None, rank: int | None = None,
                 backend: str = "nccl", timeout_s: float = 600.0):
        self.world = int(world if world is not None else os.environ.get("WORLD_SIZE", 1))
        self.rank = int(rank if rank is not None else os.environ.get("RANK", 0))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            if backend == "nccl":
                import torch
                torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", self.rank)))
            dist.init_process_group(backend, rank=self.rank, world_size=self.world,
                                    timeout=timedelta(seconds=timeout_s))
            self._dist = dist

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """The largest x over the ranks (every rank gets it)."""
        if self._dist is None:
            return float(x)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, units_per_rank: float, ms: float) -> float:
        """Whole-job rate: the units of every rank over the (slowest rank's) time in ms."""
        return units_per_rank * self.world / (ms * 1e-3)

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
