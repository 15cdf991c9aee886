"""Replica plumbing for multi-GPU runs: one process per GPU, each stepping its
own copy of a workload, or its share of a set of independent cases (deal);
the step has no exchange between GPUs, so there is no data-path
collective.  The only collectives are a barrier around timed
regions and a max over ranks of each timed duration, so a whole-job figure is
every rank's work divided by the slowest rank's time.

Ranks come from the launcher's environment (RANK, WORLD_SIZE, LOCAL_RANK, as
torchrun sets them); a single process without them is rank 0 of 1.  The group
runs over NCCL on GPUs and over gloo on CPU (the tests).
"""
from __future__ import annotations

import datetime
import os


def env_ranks():
    """(rank, world, local_rank) from the launcher's environment."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def whole_job_rate(units_per_rank: float, steps: int, ms_max: float, world: int) -> float:
    """Units per second of the whole job, in millions: every rank processed
    units_per_rank x steps units and the job took the slowest rank's time."""
    if ms_max <= 0:
        raise ValueError("non-positive duration")
    return world * units_per_rank * steps / (ms_max / 1e3) / 1e6


def deal(sizes, world: int):
    """Deals independent cases (uneven sizes: grid cells) to `world` ranks:
    largest first onto the least-loaded rank (ties to the lower rank), so
    the slowest rank carries as little as the sizes allow.  Returns a list
    of case indices per rank, each in ascending order.  Deterministic: every
    rank computes the same deal without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += sizes[i]
    return [sorted(x) for x in out]


class ReplicaGroup:
    """Barrier and max-over-ranks for replica runs.  backend: "nccl" (tensors
    on the local GPU) or "gloo" (CPU tensors)."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0):
        self.rank, self.world, self.local = env_ranks()
        self.backend = backend
        self.dist = self.world > 1
        self._torch = None
        if self.dist:
            import torch
            import torch.distributed as td
            self._torch = torch
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self) -> None:
        if self.dist:
            self._torch.distributed.barrier()

    def max_over_ranks(self, x: float) -> float:
        if not self.dist:
            return float(x)
        t = self._torch.tensor([float(x)], dtype=self._torch.float64, device=self._device())
        self._torch.distributed.all_reduce(t, op=self._torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.dist:
            self._torch.distributed.barrier()
            self._torch.distributed.destroy_process_group()
            self.dist = False


class LocalGroup:
    """The group of a single process (rank 0 of 1): barrier and max are
    no-ops; used where no process group was set up."""

    rank, world, local, dist = 0, 1, 0, False

    def barrier(self) -> None:
        pass

    def max_over_ranks(self, x: float) -> float:
        return float(x)

    def close(self) -> None:
        pass
