"""Multi-GPU forms of the hot path, one process per GPU.

* Independent assemblies (weak scaling): each rank builds the graph of its own
  assemblies, with no collective on the data path; ranks meet only to time the
  job (a barrier around the timed region and the maximum of the ranks' times).
* One assembly split by rows (strong scaling, rbg_bin_graph_sharded): the
  library exchanges sketch rows, row maxima and neighbour lists through an
  allgather the caller supplies; `host_allgather` (gloo, host buffers) and
  `device_allgather` (NCCL, device buffers) wrap torch.distributed for it.

Used by bench.py under torchrun (NCCL) and by the tests (gloo).
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


def row_range(n: int, rank: int, world: int):
    """Contiguous rows [lo, hi) of rank `rank` when n rows are split evenly."""
    return n * rank // world, n * (rank + 1) // world


def host_allgather(group=None):
    """allgather(send_ptr, recv_ptr, nbytes) over host memory with
    torch.distributed (any backend that gathers CPU tensors, e.g. gloo)."""
    import ctypes
    import numpy as np
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)

    def gather(send, recv, nbytes):
        src = np.ctypeslib.as_array((ctypes.c_uint8 * nbytes).from_address(send))
        t = torch.from_numpy(src.copy())
        outs = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(outs, t, group=group)
        dst = np.ctypeslib.as_array((ctypes.c_uint8 * (nbytes * world)).from_address(recv))
        for r, o in enumerate(outs):
            dst[r * nbytes:(r + 1) * nbytes] = o.numpy()
    return gather


class _DeviceBytes:
    """A device byte range as a CUDA array (zero-copy for torch.as_tensor)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                         "data": (ptr, False), "version": 3}


def device_allgather(group=None):
    """allgather(send_ptr, recv_ptr, nbytes) over device memory of the current
    GPU with torch.distributed (NCCL); complete when it returns."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)

    def gather(send, recv, nbytes):
        dev = torch.device("cuda", torch.cuda.current_device())
        s = torch.as_tensor(_DeviceBytes(send, nbytes), device=dev)
        r = torch.as_tensor(_DeviceBytes(recv, nbytes * world), device=dev)
        dist.all_gather_into_tensor(r, s, group=group)
        torch.cuda.synchronize(dev)
    return gather
