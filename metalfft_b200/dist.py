"""Replica helpers for running the FFT path on several GPUs of one node.

Every workload of this library shards into independent lines (transforms,
OLA blocks, SAR pulses), so N GPUs run N replicas: each rank takes its own
slice or its own batch and no collective touches the data.  The only
cross-rank operations are the barrier around a timed region and the
max-over-ranks of its time.
"""
import os


def rank_world():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(total, rank, world):
    """Contiguous slice [start, start + count) of `total` lines for `rank`;
    slices are disjoint, cover [0, total) and differ in size by at most 1."""
    base, extra = divmod(int(total), int(world))
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def replica_seed(seed, rank):
    """Seed of a rank's own synthetic batch (weak scaling)."""
    return int(seed) + int(rank)


def max_over_ranks(value, device=None):
    """Maximum of a float over the ranks of the default process group (the
    value itself when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
