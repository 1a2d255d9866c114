"""Multi-GPU plumbing of the update path: independent replicas.

One graph does not shard (every movement round reads global community degrees
and neighbour labels), so N GPUs run N independent graphs, one per rank, with
no collective on the data path.  The process group only provides a barrier
around the timed region and the maximum of the per-rank times; the whole-job
rate is N × steps × batch edges over that maximum.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """Rank context read from the torchrun environment (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_ADDR/PORT).  `backend` is "nccl" on GPUs, "gloo" on CPU."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 600):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if backend == "nccl":
                import torch
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """The largest value of x over all ranks (every rank calls this)."""
        if self.dist is None:
            return float(x)
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def whole_job_rate(self, steps: int, batch_edges: int, max_seconds: float) -> float:
        """Edge-updates/s of all replicas together: each rank applied `steps`
        batches of `batch_edges` updates; the job took the slowest rank's time."""
        return self.world * steps * batch_edges / max_seconds

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
