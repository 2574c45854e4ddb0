"""Host logic for running the step on several GPUs of one node.

The single-grid step does not shard (one simulation = one GPU): N GPUs run
independent replicas.  Batches of independent simulations do shard: each
simulation goes whole to one rank, balanced by cell count (largest first onto
the least loaded rank).  Neither needs a data-path collective; the only
collectives are for timing (max over ranks) and the final metric sums.
"""
import heapq


def shard_sims(cell_counts, world_size):
    """Assign simulations (given their cell counts) to ranks: greedy longest-
    processing-time bin packing.  Returns a list of index lists, one per rank,
    each in ascending simulation order."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    heap = [(0, r) for r in range(world_size)]
    out = [[] for _ in range(world_size)]
    for idx in sorted(range(len(cell_counts)), key=lambda i: (-cell_counts[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(idx)
        heapq.heappush(heap, (load + cell_counts[idx], r))
    return [sorted(o) for o in out]


def replica_seed(base_seed, rank):
    """Scene seed of replica `rank` (each replica advances its own scene)."""
    return base_seed + rank


def max_over_ranks(value, group=None):
    """Max of a host float over all ranks (timing: the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value, group=None):
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())
