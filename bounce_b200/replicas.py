"""Several GPUs: independent cloths partitioned over ranks, one process per GPU.

Cloths never interact, so the step has no exchange: each rank owns whole
cloths on its own GPU and steps them with the single-GPU path (no collective
in the step).  Collectives appear only around it, for planning checks and
for timing (the max over ranks of each rank's device time).

The partition is the longest-processing-time rule: cloths in decreasing
order of work (vertices), each to the rank with the least work so far, ties
to the lowest rank.  It is a pure function of the cloth sizes, so every rank
computes the same plan without communicating.  An optional per-rank HBM
budget (bytes of resident cloth state) is checked against the plan.
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class RankEnv:
    rank: int
    world: int
    local_rank: int


def rank_env() -> RankEnv:
    """RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them (1 process when unset)."""
    return RankEnv(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                   int(os.environ.get("LOCAL_RANK", "0")))


class BudgetError(ValueError):
    """A rank's share of the cloths does not fit its HBM budget."""


def plan_shards(work, world: int, bytes_of=None, budget_bytes: int | None = None) -> list[list[int]]:
    """Partition cloth indices 0..len(work)-1 over `world` ranks.

    work: per-cloth work (vertex count).  bytes_of: per-cloth resident bytes
    (defaults to work), checked against budget_bytes per rank when given.
    Returns one ascending index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    work = [int(w) for w in work]
    if any(w < 0 for w in work):
        raise ValueError("negative work")
    size = list(work) if bytes_of is None else [int(b) for b in bytes_of]
    if len(size) != len(work):
        raise ValueError("bytes_of and work differ in length")
    order = sorted(range(len(work)), key=lambda k: (-work[k], k))
    load = [0] * world
    used = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(k)
        load[r] += work[k]
        used[r] += size[k]
    if budget_bytes is not None:
        for r in range(world):
            if used[r] > budget_bytes:
                raise BudgetError(f"rank {r} needs {used[r]} bytes, budget {budget_bytes}")
    return [sorted(s) for s in shards]


def shard_loads(work, shards) -> list[int]:
    """Total work of each rank's shard."""
    return [sum(int(work[k]) for k in s) for s in shards]


def _reduce(value: float, op: str) -> float:
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    backend = dist.get_backend()
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op={"max": dist.ReduceOp.MAX, "sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN}[op])
    return float(t.item())


def max_over_ranks(value: float) -> float:
    """The largest value over all ranks (device times: the job takes as long as its slowest rank)."""
    return _reduce(value, "max")


def sum_over_ranks(value: float) -> float:
    return _reduce(value, "sum")


def aggregate_rate(units: float, seconds: float) -> float:
    """Whole-job rate: the units all ranks processed over the slowest rank's time."""
    total = sum_over_ranks(units)
    slowest = max_over_ranks(seconds)
    return total / slowest if slowest > 0 else 0.0


def check_same_plan(shards) -> bool:
    """True when every rank computed the same partition (a cheap digest compared with a MIN/MAX pair)."""
    digest = 0
    for r, s in enumerate(shards):
        for k in s:
            digest = (digest * 1000003 + (r + 1) * 7919 + k) % (1 << 50)
    return max_over_ranks(digest) == _reduce(digest, "min")
