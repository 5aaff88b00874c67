"""Replica plumbing for running one solver per GPU (torch.distributed).

The PDHG path does not shard: a single LP would need an all-gather of the
iterates every iteration, and the path has no exchange step. Multi-GPU runs
are therefore replicas (each rank solves its own instance, weak scaling), and
the only collectives are the ones that time and report the job: a barrier
around the timed region, the maximum of the ranks' times, and the sum of the
units they processed. One process per GPU with NCCL over NVLink on GPUs; gloo
on CPU (the tests). Every rank takes the same collective steps in the same
order; the process group has a short timeout so that a rank that never
arrives ends the others' collectives with an error.
"""

from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    world: int
    rank: int
    local: int
    backend: str | None  # None: one process, no process group

    @property
    def device(self) -> str:
        return f"cuda:{self.local}" if self.backend == "nccl" else "cpu"


def init(backend: str | None = None, timeout_s: float = 600.0) -> Ranks:
    """Reads WORLD_SIZE / RANK / LOCAL_RANK (torchrun's environment) and, for
    more than one rank, joins the process group: NCCL with this rank's GPU
    when CUDA is there (unless `backend` says otherwise), else gloo."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws <= 1:
        return Ranks(1, 0, 0, None)
    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return Ranks(ws, rank, local, backend)


def barrier(r: Ranks) -> None:
    if r.backend is not None:
        import torch.distributed as dist
        dist.barrier()


def _reduce(r: Ranks, v: float, op_name: str) -> float:
    if r.backend is None:
        return float(v)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=r.device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(r: Ranks, v: float) -> float:
    """The largest of the ranks' values (a job's time is its slowest rank's)."""
    return _reduce(r, v, "MAX")


def sum_over_ranks(r: Ranks, v: float) -> float:
    return _reduce(r, v, "SUM")


def whole_job_rate(r: Ranks, units: float, seconds: float) -> tuple[float, float]:
    """(units all ranks processed / the slowest rank's seconds, that time)."""
    t = max_over_ranks(r, seconds)
    total = sum_over_ranks(r, units)
    return total / t, t


def finish(r: Ranks) -> None:
    """Final barrier and leaving the process group (every rank calls it)."""
    if r.backend is not None:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
