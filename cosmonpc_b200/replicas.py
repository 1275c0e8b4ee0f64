"""Replica data parallelism: independent data vectors (mocks, catalogs) sharded
over ranks, one process per GPU, no data-path collective.

The mesh estimator has no exchange step between catalogs: each rank computes
whole data vectors of its own units and the job's throughput is the units of
every rank over the slowest rank's time.  The only collectives are the
barrier around a timed region and a MAX of the per-rank times (the reference
reaches the same independence with one MPI job per catalog).
"""
from __future__ import annotations

import os


def rank_info():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_units, rank, world):
    """Contiguous block of unit indices owned by ``rank`` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d out of range for world size %d" % (rank, world))
    base, extra = divmod(int(n_units), world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def unit_seed(base_seed, unit):
    """Seed of unit ``unit`` (the same on every rank layout, so sharded and serial runs agree)."""
    return int(base_seed) + int(unit)


def max_over_ranks(x, device=None):
    """MAX of a per-rank float over the default process group (x itself without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    if device is None:
        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, seconds, world):
    """Whole-job throughput: units of all ranks over the slowest rank's seconds."""
    return units_per_rank * world / seconds
