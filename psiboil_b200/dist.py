"""Multi-GPU plumbing: one process per GPU, independent problems per rank.

The pressure solves of a batch (or of a serving stream) are independent, so
ranks share no data during a solve: a batch is split across ranks by cost
(cells), each rank solves its share on its own GPU, and only the timing and
the per-problem results travel, through torch.distributed (NCCL on GPUs,
gloo on CPU). There is no collective inside a solve.
"""
import heapq

import torch
import torch.distributed as dist


def shard_by_cost(costs, world):
    """Deterministic longest-processing-time assignment of problems to ranks.

    costs: per-problem cost (e.g. cell count). Returns a list, one entry per
    problem, of the rank that solves it; ties break by problem index and
    rank, so every rank computes the same assignment without communication.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return owner


def my_share(costs, rank, world):
    """Indices of the problems rank `rank` solves."""
    owner = shard_by_cost(costs, world)
    return [i for i, r in enumerate(owner) if r == rank]


def _device():
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(value):
    """Maximum of a float over all ranks (the job's time is the slowest rank's)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value):
    """Sum of a float over all ranks (work done by the whole job)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_results(local):
    """All ranks' per-problem results as one dict {problem index: result}.

    local: dict {problem index: picklable result} of this rank."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, dict(local))
    merged = {}
    for part in out:
        merged.update(part)
    return merged
