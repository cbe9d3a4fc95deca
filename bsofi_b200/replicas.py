"""Multi-GPU execution of independent BSOF/I inversions: replicas.

Independent inversions (Monte Carlo walkers, serving requests) shard by
instance across ranks, one process per GPU, with no collective on the data
path; the only collectives are a barrier around timed regions and a MAX
reduction of the elapsed device time, so throughput is "all instances /
slowest rank".  (Splitting one inversion across the GPUs of a group is a
separate path, bsofi_b200.shard.)
"""
import os


def world():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(count, rank, world_size):
    """Instance indices owned by `rank`: a contiguous balanced block."""
    base, extra = divmod(count, world_size)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return list(range(lo, hi))


def shard_by_cost(costs, rank, world_size):
    """Greedy longest-processing-time assignment of instances to ranks;
    every rank computes the same assignment and keeps its own part."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world_size
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def max_over_ranks(value, device=None):
    """MAX of a float over the process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
