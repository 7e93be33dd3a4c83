"""The ProbMinHash4 query surface on the device against the reference's own
ProbMinHash4 (src/probmh.h:103-283): per-contig winners and register values
(getWinners / getRegisters of the sketch build_pmh_winners makes), the
many-vs-many jaccard_weighted / jaccard / distance / ani, and merge.  Every
value must be bit-identical.

With RABBIT_GC_NORM=0 a contig's elements are its canonical 4-mers in
ascending code order with weight count / total (src/rabbitbin.cpp:1486-1490),
so the reference sketch can be rebuilt here from the sequence alone.
"""
import numpy as np
import pytest

from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly

pytestmark = pytest.mark.gpu

_LUT = np.full(256, 255, np.uint8)
for _c, _v in zip(b"ACGTacgt", [0, 1, 2, 3, 0, 1, 2, 3]):
    _LUT[_c] = _v


def _elements(seq, k=4):
    """(ascending canonical k-mer codes, weights) of one contig, gc-norm 0."""
    mask, hs = (1 << (2 * k)) - 1, 2 * (k - 1)
    counts = np.zeros(1 << (2 * k), np.int64)
    fwd = rev = valid = 0
    for b in _LUT[np.frombuffer(seq, np.uint8)]:
        if b == 255:
            fwd = rev = valid = 0
            continue
        fwd = ((fwd << 2) | int(b)) & mask
        rev = (rev >> 2) | ((3 ^ int(b)) << hs)
        valid += 1
        if valid >= k:
            counts[min(fwd, rev)] += 1
    total = int(counts.sum())
    codes = np.nonzero(counts)[0].astype(np.uint64)
    inv = 1.0 / float(total) if total else 0.0
    return codes, counts[counts > 0].astype(np.float64) * inv


def _contigs(seed, n):
    asm = make_assembly(6, n, 0, seed=seed, median_len=1200.0, min_len=300, max_len=4000,
                        n_frac=0.01)
    seqs = [b"", b"ACG", b"NNNNNNNN", b"ACGT" * 20] + asm.seqs
    offs = np.zeros(len(seqs) + 1, np.int64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    return seqs, b"".join(seqs), offs


def test_sketch_rows_against_reference(gpu_ctx, ref_lib):
    seqs, buf, offs = _contigs(301, 50)
    w64, regs = gpu_ctx.build_pmh_sketches(buf, offs, api.default_params(gc_norm=0))
    for i, s in enumerate(seqs):
        codes, wts = _elements(s)
        r_ref, w_ref = ref_lib.pmh_elements(codes, wts, m=500)
        assert np.array_equal(w64[i], w_ref), f"contig {i}: winners differ"
        assert np.array_equal(regs[i], r_ref), f"contig {i}: registers differ"
    # default GC norm: the 64-bit winners fold to the reference's 32-bit rows
    w64, _ = gpu_ctx.build_pmh_sketches(buf, offs)
    w32 = (w64 ^ (w64 >> np.uint64(32))).astype(np.uint32)
    assert np.array_equal(w32, ref_lib.build_winners(buf, offs))


def test_compare_metrics_against_reference(gpu_ctx, ref_lib):
    seqs, buf, offs = _contigs(302, 40)
    w64, regs = gpu_ctx.build_pmh_sketches(buf, offs, api.default_params(gc_norm=0))
    ia, ib = list(range(0, 18)), list(range(14, 44))      # overlapping sets: self pairs too
    got = {m: gpu_ctx.pmh_compare(m, (w64 if m == "jaccard_weighted" else regs)[ia],
                                  (w64 if m == "jaccard_weighted" else regs)[ib])
           for m in ("jaccard_weighted", "jaccard", "distance", "ani")}
    els = [_elements(s) for s in seqs]
    for x, i in enumerate(ia):
        for y, j in enumerate(ib):
            want = ref_lib.pmh_metrics(els[i][0], els[i][1], els[j][0], els[j][1], m=500)
            for m, v in zip(("jaccard_weighted", "jaccard", "distance", "ani"), want):
                g = got[m][x, y]
                assert g == v or (np.isinf(g) and np.isinf(v)), (m, i, j, g, v)


def test_merge_registers(gpu_ctx):
    seqs, buf, offs = _contigs(303, 30)
    _, regs = gpu_ctx.build_pmh_sketches(buf, offs)
    a, b = regs[:17], regs[17:34]
    got = gpu_ctx.pmh_merge_registers(a, b)
    assert np.array_equal(got, np.where(b < a, b, a))


def test_compare_rejects_bad_arguments(gpu_ctx):
    with pytest.raises(api.RbgError):
        gpu_ctx.pmh_compare("jaccard", np.zeros((2, 1)), np.zeros((2, 1)))
