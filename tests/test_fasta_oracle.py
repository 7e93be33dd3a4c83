"""FASTA ingest oracle: the restated parser against RabbitBin's own
parse_fasta_mmap_parallel (compiled into the reference harness) on seeded
random files with the awkward cases real assemblies carry: line wrapping at
any width, CRLF, blank lines, '>' inside sequence lines, spaces and tabs,
lower case and IUPAC codes, empty bodies, junk before the first record, and a
last header without a newline."""
import os
import tempfile

import numpy as np
import pytest

import oracle


def random_fasta(seed, n_rec=40):
    rng = np.random.default_rng(seed)
    out = []
    if rng.random() < 0.3:
        out.append(b"junk before the first record\n")
    alphabet = np.frombuffer(b"ACGTACGTACGTacgtNRY", dtype=np.uint8)
    for r in range(n_rec):
        name = b"ctg%d" % r
        sep = bytes(rng.choice([b" ", b"\t"])) if rng.random() < 0.5 else b""
        desc = sep + b"len=%d x>y" % r if sep else b""
        eol = b"\r\n" if rng.random() < 0.2 else b"\n"
        out.append(b">" + name + desc + eol)
        L = int(rng.choice([0, 5, 900, 1000, 1500, 2499, 2500, 4000, 12000]))
        seq = bytes(rng.choice(alphabet, size=L))
        if rng.random() < 0.05 and L > 10:
            seq = seq[:5] + b" " + seq[6:]
        width = int(rng.choice([0, 60, 61, 80, 4000]))
        if width == 0 or L == 0:
            lines = [seq]
        else:
            lines = [seq[i:i + width] for i in range(0, L, width)]
        body = b""
        for ln in lines:
            body += ln + eol
            if rng.random() < 0.02:
                body += eol                          # blank line
        if rng.random() < 0.03 and len(body) > 20:
            k = len(body) // 2                       # a '>' inside a sequence line
            body = body[:k] + b">" + body[k:]
        out.append(body)
    data = b"".join(out)
    if rng.random() < 0.3:
        data += b">last_without_newline"
    return data


@pytest.mark.parametrize("seed", range(30))
def test_restated_parser_matches_reference(seed):
    data = random_fasta(seed)
    with tempfile.TemporaryDirectory() as d:
        fn = os.path.join(d, "a.fa")
        with open(fn, "wb") as f:
            f.write(data)
        want = oracle.parse_fasta_ref(fn, min_contig=2500, min_small=1000, nthreads=3)
    if want is None:
        pytest.skip("reference harness not built")
    got = oracle.parse_fasta_restated(data, min_contig=2500, min_small=1000)
    assert got == want


def test_restated_parser_on_synthetic_assembly(tmp_path):
    from rabbitbin_b200.synth import make_assembly, write_fasta
    a = make_assembly(4, 60, 0, seed=5, n_small=20)
    fn = str(tmp_path / "asm.fa")
    write_fasta(a, fn)
    data = open(fn, "rb").read()
    got = oracle.parse_fasta_restated(data)
    assert [s for _, s in got["large"]] == list(a.seqs)
    assert [s for _, s in got["small"]] == [s for s in a.small_seqs if len(s) >= 1000]
    want = oracle.parse_fasta_ref(fn)
    if want is not None:
        assert got == want
