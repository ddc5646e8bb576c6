"""Multi-GPU plumbing for the paths that shard without a data-path
collective (one process per GPU, torch.distributed for the control plane).

* Replicas: every rank integrates its own Ks realisation of the same
  problem; the job's throughput is the ranks' simulated seconds over the
  slowest rank's device time.
* Ensemble members: the independent members of a batched ensemble are
  dealt to ranks by cost (node count), largest first onto the least-loaded
  rank, so ranks finish together; no member is split.

Only timings and statistics cross ranks (an all-reduce of one number, an
all-gather of small host lists).  Works with the nccl backend on GPUs and
the gloo backend on CPUs."""
from __future__ import annotations

import heapq


def replica_seed(base: int, rank: int) -> int:
    """Ks-field seed of a rank's replica"""
    return base + rank


def partition_members(costs, world_size: int):
    """largest-cost-first assignment of members to ranks; returns, per
    rank, the ascending list of member indices.  Deterministic: ties go to
    the lower rank and the lower member index."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda m: (-costs[m], m))
    heap = [(0, r) for r in range(world_size)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world_size)]
    for m in order:
        load, r = heapq.heappop(heap)
        parts[r].append(m)
        heapq.heappush(heap, (load + costs[m], r))
    return [sorted(p) for p in parts]


def max_over_ranks(x: float, device="cpu") -> float:
    """the largest value of x over all ranks (1 rank: x)"""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(sim_seconds_per_rank: float, world_size: int, max_device_seconds: float) -> float:
    """whole-job simulated seconds per wall second: every rank simulates the
    same horizon; the job takes as long as its slowest rank"""
    return sim_seconds_per_rank * world_size / max_device_seconds
