"""Process-per-GPU plumbing of the multi-GPU runs: every rank runs its own
transforms (replicas, no collective on the data path) and the timing is the
maximum over ranks.  torch.distributed carries only the timing reduction
(NCCL on GPUs, gloo for the CPU tests)."""
import os

__all__ = ["dist_env", "max_over_ranks", "job_seconds_per_transform",
           "split_range"]


def dist_env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(value, device=None):
    """The maximum of `value` over all ranks of the default process group
    (the value itself without one).  Every rank must call it."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_seconds_per_transform(max_seconds, steps, world):
    """Whole-job time per transform: `world` replicas each ran `steps`
    transforms in at most `max_seconds`."""
    if steps <= 0 or world <= 0:
        raise ValueError("steps and world must be positive")
    return max_seconds / (steps * world)


def split_range(n, rank, world):
    """Contiguous share [lo, hi) of n independent items for `rank` of
    `world` (sizes differ by at most one)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)
