"""One process per GPU: the rank plumbing of multi-GPU runs.

Two multi-GPU forms use it: one tangle over all ranks (openvort_b200.shard,
whose exchange is an all-gather of the Biot-Savart sums), and one
independent tangle per rank (no collective on the data path).  Beyond that
exchange the collectives are the timing ones: a barrier around the timed
region and the maximum of the per-rank device times.  NCCL on GPUs, gloo on
CPU (tests).
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
    pg: object = None          # torch.distributed, or None for a single process
    device: str = "cpu"

    @property
    def is_root(self) -> bool:
        return self.rank == 0


def setup(backend: str | None = None, timeout_s: float = 600.0) -> Ranks:
    """Read RANK / LOCAL_RANK / WORLD_SIZE (torchrun) and, when WORLD_SIZE > 1,
    join the process group: NCCL with this rank's GPU, else gloo."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Ranks(1, 0, local)
    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    device = "cpu"
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
        device = f"cuda:{local}"
    dist.init_process_group(backend, **kw)
    return Ranks(world, rank, local, dist, device)


def describe(r: Ranks) -> dict:
    """The process group as the run saw it: backend, world size and, for
    NCCL, the library version torch loaded."""
    if r.pg is None:
        return {"backend": None, "world": 1}
    out = {"backend": r.pg.get_backend(), "world": r.pg.get_world_size()}
    if out["backend"] == "nccl":
        import torch
        v = torch.cuda.nccl.version()
        out["nccl_version"] = ".".join(map(str, v)) if isinstance(v, tuple) else str(v)
    return out


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank r's own tangle (independent tangles per rank)."""
    return seed + 1000 * rank


def max_over_ranks(r: Ranks, x: float) -> float:
    if r.pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=r.device)
    r.pg.all_reduce(t, op=r.pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(r: Ranks, x: float) -> float:
    if r.pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=r.device)
    r.pg.all_reduce(t, op=r.pg.ReduceOp.SUM)
    return float(t.item())


def barrier(r: Ranks):
    """All ranks here, and (on GPUs) this rank's device idle."""
    if r.pg is not None:
        r.pg.barrier()
    if r.device.startswith("cuda"):
        import torch
        torch.cuda.synchronize()


def close(r: Ranks):
    if r.pg is not None:
        r.pg.destroy_process_group()
