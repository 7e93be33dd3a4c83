"""One-permutation MinHash (the RABBIT_PMH=0 metric of rabbit_sketch.h): the
CPU restatement of KmerSketch update / densify / buildSig against the
reference's own header compiled in the harness, bucket for bucket."""
import numpy as np
import pytest


def _fuzz(seed):
    rng = np.random.default_rng(seed)
    alpha = np.frombuffer(b"ACGTacgtNRY-", np.uint8)
    p = np.array([.22, .22, .22, .22, .02, .02, .02, .02, .02, .01, .005, .005])
    seqs = [rng.choice(alpha, p=p / p.sum(), size=int(L)).astype(np.uint8).tobytes()
            for L in [0, 1, 5, 8, 31, 32, 33, 100, 2500, 7000, 20000]]
    seqs += [b"N" * 50, b"A" * 64, b"ACGT" * 40, b"acgtn" * 30]
    offs = np.zeros(len(seqs) + 1, np.int64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    return b"".join(seqs), offs


@pytest.mark.parametrize("m,K,bits", [(500, 8, 2), (2, 1, 1), (64, 4, 1), (130, 15, 3),
                                      (1000, 21, 2), (4096, 12, 2), (250, 32, 7)])
def test_restated_oph_matches_reference(ref_lib, orc, m, K, bits):
    cat, offs = _fuzz(m + K)
    want = ref_lib.oph_values(cat, offs, m, K, bits)
    got = orc.oph_values(cat, offs, m, K, bits)
    assert np.array_equal(got, want)
    assert want.max() < (1 << bits)
    # contigs without a valid k-mer have the all-zero signature
    lens = np.diff(offs)
    assert not want[lens < K].any()
