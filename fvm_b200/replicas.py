"""One process per GPU for the multi-GPU runs.

The single-mesh solve does not shard (no partitioned path is built), so N
GPUs run N independent replicas of it. A batch of independent meshes does
shard: each rank solves its own subset, chosen by greedy bin-packing on cell
counts, with no exchange at all on the data path. The ranks only agree on
their timings (the maximum over ranks) through the process group: NCCL on
GPUs, gloo on the host (tests).

Launch as `torchrun --nproc-per-node N ...` (RANK, LOCAL_RANK, WORLD_SIZE,
MASTER_ADDR, MASTER_PORT in the environment); with WORLD_SIZE unset or 1
everything is local and no process group is created.
"""
from __future__ import annotations

import datetime
import os


class Ranks:
    def __init__(self, backend: str | None = None, timeout_s: float = 600.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist

            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = "cuda"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = dist
            self.torch = torch

    def barrier(self) -> None:
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        """The maximum of v over all ranks (every rank gets it)."""
        if not self.pg:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self) -> None:
        if self.pg:
            self.pg.destroy_process_group()
            self.pg = None


def shard_meshes(cells, world: int, rank: int) -> list[int]:
    """Indices of the meshes rank `rank` of `world` solves: meshes taken
    largest first (ties by index), each to the least-loaded rank (ties to the
    lower rank). Deterministic; every mesh goes to exactly one rank, and no
    rank's load exceeds the average by more than the largest mesh."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    order = sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i))
    load = [0] * world
    owner = [0] * len(cells)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += int(cells[i])
    return [i for i in range(len(cells)) if owner[i] == rank]
