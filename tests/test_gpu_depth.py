"""BAM -> depth summariser on the device against the reference's own code.

The device path (host BGZF inflation and record walk, one device thread per
record, means on the device) must give the reference's per-contig depth sums
exactly (integers) and its means bit for bit (each mean is one IEEE double
division rounded to float, src/rabbit_depth.cpp:1515-1534).  The sums come
from tests/golden/depth.npz (made by the reference's depth_accumulate_sample,
tests/golden/make_depth_golden.py) or from that code itself
(oracle/_ref/librbref_depth.so) for cases beyond the fixture."""
import gzip
import os
import struct

import numpy as np
import pytest

import oracle
from depth_cases import CASES, PARAMS, case
from rabbitbin_b200 import api
from rabbitbin_b200.synth import bam_records, make_bam

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "depth.npz"))


def _kw(pid, edge, inc, mq, dq, **extra):
    return dict(percent_identity=pid, max_edge_bases=edge, include_edge_bases=int(inc),
                min_map_qual=mq, dual_map_qual=dq, **extra)


def _check_means(out, tl, edges, min_len=1):
    kept = np.nonzero(tl.astype(np.int64) >= min_len)[0]
    np.testing.assert_array_equal(out["tid"], kept)
    np.testing.assert_array_equal(out["lens"], tl[kept].astype(np.int32))
    for c, e in enumerate(edges):
        want = oracle.depth_means(out["sums"][c], tl, e)[kept]
        np.testing.assert_array_equal(out["means"][:, c], want, err_msg=f"column {c}")


@pytest.mark.parametrize("route", ["device", "host"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_bam_depth_matches_reference(gpu_ctx, golden, name, route):
    """Both routes: BGZF inflated on the device (files whose records cross
    block ends fall back to the host walk) or on the host threads."""
    lens, _, bam = case(name)
    for i, (pid, edge, inc, mq, dq) in enumerate(PARAMS):
        out = gpu_ctx.bam_depth([bam], device_inflate=int(route == "device"),
                                **_kw(pid, edge, inc, mq, dq))
        straddle = CASES[name][2].get("straddle", False)
        assert out["device_bams"] == (1 if route == "device" and not straddle else 0)
        avg = int(golden[f"{name}/{i}/avg"])
        assert out["avg_read"][0] == avg
        np.testing.assert_array_equal(out["sums"][0], golden[f"{name}/{i}/sums"],
                                      err_msg=f"{name} params {i}")
        if dq:
            np.testing.assert_array_equal(out["sums"][1], golden[f"{name}/{i}/sums_u"])
        e = 0 if inc else min(edge, avg // 3)
        _check_means(out, lens, [e] * out["sums"].shape[0])
        assert out["names"][:3] == [f"contig_{t}" for t in out["tid"][:3]]


def test_small_chunks_carry_records_and_sample_read_length(gpu_ctx, golden):
    """1 MiB hand-overs: records cut by every chunk end, and fewer than 4,000
    mapped records in the first chunk (the read-length sample spans chunks);
    on the device route, chunks of 1 MiB of blocks (many launches per file)."""
    for name in ("edge_mix", "edge_mix_straddle", "long_reads"):
        lens, _, bam = case(name)
        for dev in (0, 1):
            out = gpu_ctx.bam_depth([bam], chunk_mb=1, device_chunk_mb=1, threads=3,
                                    device_inflate=dev, **_kw(*PARAMS[0]))
            np.testing.assert_array_equal(out["sums"][0], golden[f"{name}/0/sums"])
            assert out["avg_read"][0] == int(golden[f"{name}/0/avg"])


def test_several_bams_and_dual_columns(gpu_ctx, golden):
    lens, _, b0 = case("edge_mix")
    depth = np.random.default_rng(9).uniform(0.2, 25.0, len(lens))
    b1 = make_bam(lens, depth, seed=99, read_len=100)
    b2 = make_bam(lens, depth * 0.3, seed=98, read_len=250, straddle=True)
    pid, edge, inc, mq, dq = PARAMS[1]
    out = gpu_ctx.bam_depth([b0, b1, b2], min_contig_length=1000, **_kw(pid, edge, inc, mq, dq))
    assert out["sums"].shape == (6, len(lens))
    edges = []
    for b, bam in enumerate((b0, b1, b2)):
        recs, tl, _ = bam_records(bam)
        want = oracle.depth_accumulate_ref(recs, tl, pid, edge, inc, mq)
        if want is None:
            pytest.skip("reference harness not built")
        np.testing.assert_array_equal(out["sums"][b], want[0])
        assert out["avg_read"][b] == want[1]
        want_u = oracle.depth_accumulate_ref(recs, tl, pid, edge, inc, max(mq, dq))[0]
        np.testing.assert_array_equal(out["sums"][3 + b], want_u)
        edges.append(min(edge, want[1] // 3))
    _check_means(out, lens, edges + edges, min_len=1000)


def test_records_entry_point(gpu_ctx, golden):
    for name in ("edge_mix", "all_overhang"):
        lens, _, bam = case(name)
        recs, tl, _ = bam_records(bam)
        pid, edge, inc, mq, dq = PARAMS[1]
        s, su, avg = gpu_ctx.depth_accumulate(recs, tl, chunk_mb=2, **_kw(pid, edge, inc, mq, dq))
        np.testing.assert_array_equal(s, golden[f"{name}/1/sums"])
        np.testing.assert_array_equal(su, golden[f"{name}/1/sums_u"])
        assert avg == int(golden[f"{name}/1/avg"])


def test_paths_and_empty_files(gpu_ctx, golden, tmp_path):
    lens, _, bam = case("clean")
    p = tmp_path / "a.bam"
    p.write_bytes(bam)
    out = gpu_ctx.bam_depth([str(p)], **_kw(*PARAMS[0]))
    np.testing.assert_array_equal(out["sums"][0], golden["clean/0/sums"])
    # contigs without reads, and a file with no records at all
    empty = make_bam(np.array([1000, 2000], np.uint32), np.zeros(2), n_unmapped_tail=0)
    out = gpu_ctx.bam_depth([empty])
    assert out["records"] == 0 and out["avg_read"][0] == 0
    np.testing.assert_array_equal(out["sums"][0], [0, 0])
    np.testing.assert_array_equal(out["means"][:, 0], [0, 0])


def _blocks(bam):
    o, out = 0, []
    while o < len(bam):
        bsize = struct.unpack_from("<H", bam, o + 16)[0] + 1
        out.append((o, bsize))
        o += bsize
    return out


def test_malformed_input_is_rejected(gpu_ctx):
    lens, _, bam = case("few_reads")
    blocks = _blocks(bam)
    bad = []
    bad.append(b"not a bam file at all" * 4)
    bad.append(bam[:blocks[1][0] + 30])                       # cut inside a block
    o, n = blocks[1]
    crc = bytearray(bam)
    crc[o + n - 6] ^= 0xFF                                     # CRC32 of block 1
    bad.append(bytes(crc))
    # a record whose block_size runs past the end of the stream
    raw = gzip.decompress(bam)
    body = bytearray(raw)
    hdr_end = len(raw) - len(bam_records(bam)[0])
    struct.pack_into("<i", body, hdr_end, 10 ** 6)
    import zlib
    c = zlib.compressobj(6, zlib.DEFLATED, -15)
    cdata = c.compress(bytes(body)) + c.flush()
    assert len(body) < 65280
    blk = (b"\x1f\x8b\x08\x04\0\0\0\0\0\xff\x06\0BC\x02\0" + struct.pack("<H", 18 + len(cdata) + 8 - 1)
           + cdata + struct.pack("<II", zlib.crc32(bytes(body)), len(body)))
    bad.append(blk)
    for b in bad:
        for dev in (0, 1):
            with pytest.raises(api.RbgError) as e:
                gpu_ctx.bam_depth([b], device_inflate=dev)
            assert e.value.code == -1
    other = make_bam(np.array([300, 401], np.uint32), np.ones(2))
    with pytest.raises(api.RbgError) as e:
        gpu_ctx.bam_depth([bam, other])
    assert e.value.code == -1
    # the context still works afterwards
    out = gpu_ctx.bam_depth([bam])
    assert out["records"] > 0


def test_depth_table_from_device_sums(gpu_ctx):
    """The TSV of compute_depth_tsv_inmem from the device route's sums
    (rbg_depth_tsv), byte for byte against the reference's printDepthTable fed
    the reference's own sums."""
    lens, _, b0 = case("edge_mix")
    b1 = make_bam(lens, np.random.default_rng(4).uniform(0.2, 25.0, len(lens)), seed=77,
                  read_len=100)
    names = ["x/s1.bam", "y/s2.bam"]
    sums, avg = [], []
    for bam in (b0, b1):
        recs, tl, _ = bam_records(bam)
        want = oracle.depth_accumulate_ref(recs, tl)
        if want is None:
            pytest.skip("reference harness not built")
        sums.append(want[0])
        avg.append(want[1])
    for variance in (False, True):
        out = gpu_ctx.bam_depth([b0, b1], tsv_names=names, tsv_variance=variance)
        assert out["device_bams"] == 2
        ref = oracle.depth_tsv_ref(np.stack(sums), avg, lens,
                                   [f"contig_{i}" for i in range(len(lens))], names, variance)
        assert out["tsv"] == ref
