"""Multi-GPU form of the hot path: one process per GPU, each rank builds the
graph of its own assemblies (the path shards over independent assemblies, so
the data path has no collective).  Ranks meet only to time the job: a barrier
before and after the timed region and the maximum of the ranks' times.

Used by bench.py under torchrun (NCCL) and by the CPU tests (gloo).
"""
import datetime
import os

SEED_STRIDE = 1  # rank r of a job with base seed s builds the assembly of seed s + r


def env_rank():
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_seed(base_seed: int, rank: int) -> int:
    """Seed of the assembly rank `rank` processes."""
    return base_seed + SEED_STRIDE * rank


def init(world: int, backend: str, timeout_s: float = 600.0):
    """Process group for the timing collectives (none when world == 1)."""
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The largest of the ranks' values (every rank gets it)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Units of all ranks per second of the slowest rank (weak scaling)."""
    return units_per_rank * world / seconds


def finish(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
