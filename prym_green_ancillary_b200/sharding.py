"""Multi-GPU plumbing of the sequence stage: one process per GPU, no collective
on the data path.

The path shards by independent units (sectors, deformation operators, seeded
synthetic sequences), as the reference's pipeline does at process level
(scripts/reproduce.py: one sequence job per sector and device).  Ranks only
meet for timing: a barrier before the timed region and the maximum of the
ranks' times after it.
"""
import os


def world():
    """(rank, world_size, local_rank) from the launcher's environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def rank_seed(seed, rank, stride=1000):
    """Seed of this rank's own synthetic sequence (rank 0 keeps the base seed)."""
    return seed + stride * rank


def assign_sectors(n_sectors, world_size, rank):
    """Round-robin share of the sectors 0..n_sectors-1 for this rank (disjoint, covering)."""
    return list(range(rank, n_sectors, world_size))


def max_over_ranks(values, device=None):
    """Element-wise maximum of a list of floats over all ranks (identity for one process).

    Uses torch.distributed (NCCL on GPUs, gloo on CPU); every rank must call it
    with the same number of values.
    """
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu().tolist()]
