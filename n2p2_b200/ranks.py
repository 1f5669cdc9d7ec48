"""Multi-GPU plumbing of the benchmark: one process per GPU, each rank
evaluates its own batch of structures (structures are independent, so the
path shards with no collective on the data path); only the timing is reduced
(max over ranks)."""
import os


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(base_seed, rank):
    """Seed of a rank's batch: every rank gets a different, reproducible set of
    structures of the same size distribution (weak scaling)."""
    return base_seed + 7919 * rank


def max_over_ranks(value, device=None):
    """Max of a float over all ranks (the job's time is its slowest rank)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
