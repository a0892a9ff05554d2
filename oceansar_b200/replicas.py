"""Replica-parallel runs: one independent scene per rank, no collective on the data path.

The raw-generation path does not shard within a scene (every pulse needs the whole 2-D
surface FFT), so multi-GPU runs are replicas: rank r simulates its own scene (seed
``base + r``).  The only communication is the timing reduction: the job's time is the
maximum over ranks of each rank's device time, and the job's throughput is the echoes of
all ranks divided by that time.  Works with any ``torch.distributed`` backend (NCCL on GPUs,
gloo for CPU tests).
"""
import torch


def replica_seed(base_seed, rank):
    return int(base_seed) + int(rank)


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (the value itself without a process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    """Sum of a float over all ranks (the value itself without a process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_throughput(units_per_rank, seconds_this_rank, device=None):
    """(throughput, max seconds): all ranks' units over the slowest rank's time."""
    import torch.distributed as dist
    world = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    t = max_over_ranks(seconds_this_rank, device)
    return float(units_per_rank) * world / t, t
