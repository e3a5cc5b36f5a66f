"""One tangle over several GPUs, one process per GPU (ov_state_shard*).

Every rank holds the whole tangle and builds the same Barnes-Hut tree at
each evaluation.  Rank r of W walks only its contiguous share of the
tree's key order, and the per-target Biot-Savart sums (6 doubles per node)
are then all-gathered in place, so every rank finishes every node.  The
walk is ~97% of an RK4 step at 1M points, so that part splits W ways.  What
each rank repeats is the tree build, the geometry and the per-node
epilogue, about 3% of the step, plus 48 bytes per node and evaluation
over NVLink.  All ranks keep identical states, equal bit for bit to a
single-GPU ov_state_run.

The exchange is torch.distributed's all_gather_into_tensor (NCCL on GPUs;
gloo on CPU, which gathers a list of views instead) into the buffer the
library packs.  The library synchronises its stream before
ov_state_shard_begin returns, and the exchange waits for its own stream
before ov_state_shard_end reads the buffer.
"""
from __future__ import annotations

import torch

from .dist import Ranks


def exchange(xbuf: torch.Tensor, ranks: Ranks, block: int) -> None:
    """In-place all-gather: rank r's block is xbuf[r*block:(r+1)*block]; on
    return every rank's xbuf holds all W blocks."""
    if ranks.world <= 1:
        return
    full = xbuf[: ranks.world * block]
    mine = full[ranks.rank * block:(ranks.rank + 1) * block]
    if full.is_cuda:
        ranks.pg.all_gather_into_tensor(full, mine)
        torch.cuda.current_stream(full.device).synchronize()
    else:
        parts = list(full.split(block))
        ranks.pg.all_gather(parts, mine.clone())


class ShardedRun:
    """RK4 steps of one DeviceState shared by all ranks of `ranks`."""

    STAGES = 4   # update_tangle, then the three stages of rk4_step

    def __init__(self, state, ranks: Ranks):
        self.st = state
        self.r = ranks
        nbytes = state.shard_bytes(ranks.world)
        self.block = nbytes // (8 * ranks.world)      # doubles per rank
        if ranks.device != "cpu":
            device = torch.device(ranks.device)
        else:
            device = torch.device("cuda", ranks.local) if torch.cuda.is_available() else torch.device("cpu")
        self.xbuf = torch.zeros(max(1, nbytes // 8), dtype=torch.float64, device=device)
        state.shard(ranks.rank, ranks.world, self.xbuf.data_ptr(), nbytes)

    def step(self, t: float, dt: float) -> None:
        for q in range(self.STAGES):
            self.st.shard_begin(q, t, dt)
            exchange(self.xbuf, self.r, self.block)
            self.st.shard_end(q, t, dt)

    def run(self, t0: float, dt: float, nsteps: int) -> None:
        t = t0
        for _ in range(nsteps):
            self.step(t, dt)
            t += dt
