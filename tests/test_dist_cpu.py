"""Multi-rank form on CPU ranks (gloo, world size 2).

The hot path shards over independent assemblies: rank r builds the graph of the
assembly with seed base + r, with no data-path collective; ranks meet only for
the timing (barrier, maximum of the ranks' times).  The graphs here come from the
oracle (CPU), since these tests run without a GPU; the sharding, seeding and
timing logic is the one bench.py runs under torchrun.
"""
import hashlib
import json
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import oracle
from rabbitbin_b200 import shard
from rabbitbin_b200.synth import make_assembly

BASE_SEED = 11


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _shard_digest(rank):
    """Digest of the graph of the assembly rank `rank` is given."""
    asm = make_assembly(6, 300, 5, seed=shard.shard_seed(BASE_SEED, rank))
    buf, offs = asm.concat()
    lib = oracle.restated()
    g = lib.run_graph(oracle.default_params(asm.n, 500, 5), lib.build_winners(buf, offs), asm.depth)
    h = hashlib.blake2b(digest_size=16)
    for a in oracle.sorted_edges(g):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest(), asm.n


def _rank_main(rank, world, port, outdir, fail_rank):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r, w, _ = shard.env_rank()
    shard.init(w, "gloo", timeout_s=30)
    if r == fail_rank:
        raise RuntimeError("rank left before the timing collective")
    digest, n = _shard_digest(r)
    shard.barrier(w)
    t = 1.0 + 0.5 * r                    # this rank's (stand-in) time
    mx = shard.max_over_ranks(t, w)
    import torch.distributed as dist
    out = [None] * w
    dist.all_gather_object(out, {"rank": r, "digest": digest, "n": n, "max": mx})
    if r == 0:
        with open(os.path.join(outdir, "ranks.json"), "w") as f:
            json.dump(out, f)
    shard.finish(w)


def test_two_ranks_shard_and_time(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path), -1), nprocs=world, join=True)
    ranks = json.load(open(tmp_path / "ranks.json"))
    assert [x["rank"] for x in ranks] == [0, 1]
    for x in ranks:
        alone, n = _shard_digest(x["rank"])
        assert x["digest"] == alone                 # a shard's graph is the same alone
        assert x["max"] == 1.5                      # every rank sees the slowest time
    assert ranks[0]["digest"] != ranks[1]["digest"]  # ranks really work on different data
    pairs = [x["n"] * (x["n"] - 1) // 2 for x in ranks]
    assert shard.whole_job_rate(pairs[0], world, 1.5) == pairs[0] * 2 / 1.5


def test_failed_rank_ends_the_job(tmp_path):
    """A rank that leaves before the timing collective makes the other rank's
    collective fail within the process-group timeout instead of hanging."""
    world = 2
    try:
        mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path), 1), nprocs=world, join=True)
    except Exception as e:                          # ProcessRaisedException / ProcessExitedException
        assert "rank left before the timing collective" in str(e) or "exit" in str(e).lower()
    else:
        raise AssertionError("the job did not report the failed rank")
    assert not (tmp_path / "ranks.json").exists()


def _gather_main(rank, world, port, outdir):
    import ctypes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    shard.init(world, "gloo", timeout_s=30)
    fn = shard.host_allgather()
    nbytes = 24
    send = (np.arange(nbytes, dtype=np.uint8) + 50 * rank).astype(np.uint8)
    recv = np.zeros(nbytes * world, np.uint8)
    fn(send.ctypes.data, recv.ctypes.data, nbytes)
    if rank == 0:
        np.save(os.path.join(outdir, "recv.npy"), recv)
    shard.finish(world)


def test_host_allgather_adapter(tmp_path):
    """The host-memory collective handed to rbg_bin_graph_sharded: rank r's
    bytes land at r * nbytes of every rank's receive buffer."""
    world = 2
    mp.spawn(_gather_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    recv = np.load(tmp_path / "recv.npy")
    want = np.concatenate([(np.arange(24) + 50 * r).astype(np.uint8) for r in range(world)])
    assert np.array_equal(recv, want)


def test_row_ranges_tile_the_assembly():
    for n in (0, 1, 7, 4000):
        for world in (1, 2, 3, 8):
            rr = [shard.row_range(n, r, world) for r in range(world)]
            assert rr[0][0] == 0 and rr[-1][1] == n
            assert all(rr[r][1] == rr[r + 1][0] for r in range(world - 1))
