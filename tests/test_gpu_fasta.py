"""Device FASTA ingest (rbg_parse_fasta, rbg_bin_fasta) against the restated
parser, itself pinned to RabbitBin's own parse_fasta_mmap_parallel on the CPU
(tests/test_fasta_oracle.py): same records, names, sequences and counts, and
the graph from FASTA bytes equals the graph from the parsed contigs."""
import numpy as np
import pytest

import oracle
from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly, write_fasta
from test_fasta_oracle import random_fasta

pytestmark = pytest.mark.gpu


def _as_pairs(part):
    seqcat, offs, names = part
    return [(names[i], seqcat[offs[i]:offs[i + 1]]) for i in range(len(names))]


@pytest.mark.parametrize("seed", range(30))
def test_device_parse_matches_oracle(gpu_ctx, seed):
    data = random_fasta(seed, n_rec=60)
    want = oracle.parse_fasta_restated(data, min_contig=2500, min_small=1000)
    got = gpu_ctx.parse_fasta(data, 2500, 1000)
    assert got["num_seqs"] == want["num_seqs"]
    assert _as_pairs(got["large"]) == want["large"]
    assert _as_pairs(got["small"]) == want["small"]


@pytest.mark.parametrize("data", [b"", b"no records at all\n", b">only_header",
                                  b">a\n", b">a\nACGT", b"\n\n>x y\r\n\r\nAC\r\nGT\r\n"])
def test_device_parse_edge_files(gpu_ctx, data):
    want = oracle.parse_fasta_restated(data, min_contig=2, min_small=1)
    got = gpu_ctx.parse_fasta(data, 2, 1)
    assert got["num_seqs"] == want["num_seqs"]
    assert _as_pairs(got["large"]) == want["large"]
    assert _as_pairs(got["small"]) == want["small"]


def test_bin_fasta_equals_bin_graph(gpu_ctx, tmp_path):
    a = make_assembly(12, 1500, 5, seed=77, n_small=300)
    fn = str(tmp_path / "asm.fa")
    write_fasta(a, fn)
    data = open(fn, "rb").read()
    parsed = gpu_ctx.parse_fasta(data)
    seqcat, offs, names = parsed["large"]
    assert seqcat == b"".join(a.seqs) and len(names) == a.n
    want = gpu_ctx.bin_graph(seqcat, offs, a.depth)
    got = gpu_ctx.bin_fasta(data, a.depth)
    assert got["b0"] == want["b0"] and got["sim_cutoff"] == want["sim_cutoff"]
    for k in ("src", "dst", "scomp", "score"):
        assert np.array_equal(got[k], want[k])
