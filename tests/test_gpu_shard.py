"""One assembly split by rows over ranks (rbg_bin_graph_sharded): the ranks'
edges, concatenated in rank order, equal rbg_bin_graph's graph of the whole
assembly.  The ranks are processes on one GPU exchanging through gloo (host
buffers); their kernels never wait on one another, so they may share the GPU."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rabbitbin_b200 import api, shard
from rabbitbin_b200.synth import make_assembly

pytestmark = pytest.mark.gpu

CASES = {
    "fused_s20": dict(asm=(30, 4000, 20, 501), split=None, params=dict(force_path=2)),
    "fused_s5_uneven": dict(asm=(30, 4000, 5, 502), split=(700,), params=dict(force_path=2)),
    "small_s10": dict(asm=(20, 3000, 10, 503), split=None, params=dict(force_path=1)),
}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _assembly(spec):
    G, N, S, seed = spec
    return make_assembly(G, N, S, seed=seed, absent_frac=0.1 if S > 2 else 0.0)


def _bounds(n, world, split):
    if split is None:
        return [shard.row_range(n, r, world) for r in range(world)]
    cuts = [0] + list(split) + [n]
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def _rank_main(rank, world, port, name, outdir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    case = CASES[name]
    asm = _assembly(case["asm"])
    buf, offs = asm.concat()
    lo, hi = _bounds(asm.n, world, case["split"])[rank]
    local = buf[offs[lo]:offs[hi]]
    ctx = api.Context(0)
    g = ctx.bin_graph_sharded(local, offs[lo:hi + 1] - offs[lo], asm.depth[lo:hi], rank, world,
                              shard.host_allgather(), params=api.default_params(**case["params"]))
    np.savez(os.path.join(outdir, f"rank{rank}.npz"), src=g["src"], dst=g["dst"],
             scomp=g["scomp"], score=g["score"], b0=g["b0"], cutoff=g["sim_cutoff"])
    ctx.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_ranks_equal_whole_graph(gpu_ctx, tmp_path, name):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), name, str(tmp_path)), nprocs=world, join=True)
    case = CASES[name]
    asm = _assembly(case["asm"])
    buf, offs = asm.concat()
    want = gpu_ctx.bin_graph(buf, offs, asm.depth, api.default_params(**case["params"]))
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    for z in parts:
        assert float(z["b0"]) == want["b0"] and float(z["cutoff"]) == want["sim_cutoff"]
    lo_hi = _bounds(asm.n, world, case["split"])
    for r, z in enumerate(parts):                       # each rank's edges leave its own rows
        if len(z["src"]):
            assert lo_hi[r][0] <= z["src"].min() and z["src"].max() < lo_hi[r][1]
    for k in ("src", "dst", "scomp", "score"):
        got = np.concatenate([z[k] for z in parts])
        assert np.array_equal(got, want[k]), k


def test_one_rank_equals_whole_graph(gpu_ctx):
    """World size 1: the collective is a copy; the sharded call equals
    rbg_bin_graph, twice in a row on the same context."""
    asm = _assembly((30, 4000, 20, 504))
    buf, offs = asm.concat()
    p = api.default_params(force_path=2)
    want = gpu_ctx.bin_graph(buf, offs, asm.depth, p)
    for _ in range(2):
        got = gpu_ctx.bin_graph_sharded(buf, offs, asm.depth, 0, 1,
                                        lambda s, r, n: ctypes.memmove(r, s, n), params=p)
        assert got["b0"] == want["b0"] and got["sim_cutoff"] == want["sim_cutoff"]
        for k in ("src", "dst", "scomp", "score"):
            assert np.array_equal(got[k], want[k]), k


def _nccl_main(rank, world, port, outdir):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    asm = _assembly((30, 4000, 20, 505))
    buf, offs = asm.concat()
    p = api.default_params(force_path=2)
    ctx = api.Context(0)
    want = ctx.bin_graph(buf, offs, asm.depth, p)
    got = ctx.bin_graph_sharded(buf, offs, asm.depth, rank, world, shard.device_allgather(),
                                device_buffers=True, params=p)
    same = got["b0"] == want["b0"] and got["sim_cutoff"] == want["sim_cutoff"] and all(
        np.array_equal(got[k], want[k]) for k in ("src", "dst", "scomp", "score"))
    open(os.path.join(outdir, "same.txt"), "w").write("1" if same else "0")
    ctx.close()
    dist.destroy_process_group()


def test_device_buffer_collective(tmp_path):
    """The NCCL adapter on device buffers (world size 1: NCCL needs one GPU per
    rank, and this run has one GPU)."""
    mp.spawn(_nccl_main, args=(1, _free_port(), str(tmp_path)), nprocs=1, join=True)
    assert (tmp_path / "same.txt").read_text() == "1"
