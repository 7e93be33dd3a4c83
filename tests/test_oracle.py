"""CPU tests of the oracle itself.

The restatement (oracle/rb_oracle.cpp) is pinned against RabbitBin's own code
compiled from the reference tree (oracle/_ref) on seeded inputs, and against the
committed golden fixtures (tests/golden/), which were produced by that same
reference build (tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

import oracle
from rabbitbin_b200.synth import make_assembly

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _edge_case_seqs():
    rng = np.random.default_rng(5)
    rnd = lambda n: bytes(rng.choice(list(b"ACGT"), size=n))
    return [b"", b"AC", b"ACGT", b"N" * 30, b"A" * 40, b"ACGT" * 50,
            rnd(900).lower(), rnd(400) + b"NN" + rnd(3) + b"N" + rnd(600),
            bytes(rng.choice(list(b"ACGTNRYacgtn-"), size=1500))]


def _concat(seqs):
    offs = np.zeros(len(seqs) + 1, np.int64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    return b"".join(seqs), offs


@pytest.mark.parametrize("m", [2, 3, 17, 500, 1000])
def test_restated_winners_match_reference(ref_lib, orc, m):
    asm = make_assembly(6, 60, 0, seed=m, n_frac=0.02)
    buf, offs = _concat(_edge_case_seqs() + asm.seqs)
    assert np.array_equal(orc.build_winners(buf, offs, m=m), ref_lib.build_winners(buf, offs, m=m))


@pytest.mark.parametrize("k,gc", [(1, 1), (2, 1), (3, 0), (4, 0), (5, 1), (6, 1),
                                  (2, 2), (3, 2), (4, 2), (6, 2)])
def test_restated_winners_k_gc(ref_lib, orc, k, gc):
    asm = make_assembly(4, 40, 0, seed=10 + k)
    buf, offs = _concat(_edge_case_seqs() + asm.seqs)
    assert np.array_equal(orc.build_winners(buf, offs, k=k, gc_norm=gc),
                          ref_lib.build_winners(buf, offs, k=k, gc_norm=gc))


def test_restated_pmh_state(ref_lib, orc):
    rng = np.random.default_rng(2)
    for _ in range(20):
        ne = int(rng.integers(1, 137))
        keys = np.sort(rng.choice(2000, size=ne, replace=False)).astype(np.uint64)
        w = rng.uniform(1e-4, 20.0, size=ne)
        r1, w1 = ref_lib.pmh_elements(keys, w, m=257)
        r2, w2 = orc.pmh_elements(keys, w, m=257)
        assert np.array_equal(r1, r2) and np.array_equal(w1, w2)


def test_unit_dot_order(ref_lib, orc):
    rng = np.random.default_rng(4)
    for S in list(range(1, 70)):
        a = rng.standard_normal(S).astype(np.float32)
        b = rng.standard_normal(S).astype(np.float32)
        assert ref_lib.unit_dot_f(a, b) == orc.unit_dot_f(a, b), S


def _cmp(res_a, res_b):
    ea, eb = oracle.sorted_edges(res_a), oracle.sorted_edges(res_b)
    assert res_a["b0"] == res_b["b0"]
    assert res_a["sim_cutoff"] == res_b["sim_cutoff"]
    for x, y in zip(ea, eb):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("S", [0, 1, 2, 5])
def test_restated_small_graph(ref_lib, orc, S):
    asm = make_assembly(12, 900, S, seed=20 + S)
    buf, offs = asm.concat()
    w = ref_lib.build_winners(buf, offs)
    p = oracle.default_params(asm.n, 500, S)
    _cmp(ref_lib.run_graph(p, w, asm.depth), orc.run_graph(p, w, asm.depth))


@pytest.mark.parametrize("S,kw", [(3, {}), (20, {}), (33, {}), (1, {}), (2, {}),
                                  (5, {"mutual": 0}), (10, {"win_bits": 32}),
                                  (10, {"abdfirst": 0}), (8, {"base_on": 0})])
def test_restated_fused_graph(ref_lib, orc, S, kw):
    asm = make_assembly(20, 2700, S, seed=40 + S, absent_frac=0.1)
    buf, offs = asm.concat()
    w = ref_lib.build_winners(buf, offs)
    p = oracle.default_params(asm.n, 500, S, force_path=2, **kw)
    _cmp(ref_lib.run_graph(p, w, asm.depth), orc.run_graph(p, w, asm.depth))


def test_golden_fixtures(orc):
    """The restatement reproduces the committed reference outputs."""
    files = sorted(f for f in os.listdir(GOLDEN) if f.endswith(".npz"))
    assert files, "golden fixtures missing"
    for f in files:
        z = np.load(os.path.join(GOLDEN, f))
        if "seqcat" not in z.files:
            continue                     # label fixtures (lpa.npz), checked in test_lpa_cpu.py
        seqcat = z["seqcat"].tobytes()
        offs = z["offsets"]
        m = int(z["m"])
        w = orc.build_winners(seqcat, offs, m=m)
        assert np.array_equal(w, z["winners32"]), f
        if "src" in z.files:
            S = int(z["S"])
            p = oracle.default_params(len(offs) - 1, m, S, force_path=int(z["force_path"]))
            res = orc.run_graph(p, w, z["depth"])
            s, d, sc, sw = oracle.sorted_edges(res)
            assert res["b0"] == float(z["b0"]) and res["sim_cutoff"] == float(z["sim_cutoff"]), f
            assert np.array_equal(s, z["src"]) and np.array_equal(d, z["dst"]), f
            assert np.array_equal(sc, z["scomp"]) and np.array_equal(sw, z["score"]), f


def test_fp64_weights_against_reference(ref_lib):
    """The FP64 edge-weight oracle against the reference's own FP32 weights:
    within 1e-6 wherever both make the same cut, and any cut they disagree on
    sits on the threshold in exact arithmetic."""
    asm = make_assembly(20, 3000, 10, seed=88, absent_frac=0.1)
    buf, offs = asm.concat()
    w = ref_lib.build_winners(buf, offs)
    for fp, S in ((2, 10), (1, 5)):
        d = asm.depth[:, :S]
        res = ref_lib.run_graph(oracle.default_params(asm.n, 500, S, force_path=fp), w, d)
        rep = oracle.fp64_report(d, res)
        assert rep["edges"] > 1000
        assert rep["max_abs_err_fp64"] <= 1e-6, rep
        assert rep["max_margin_disagreeing"] <= 1e-6, rep


def test_scale_digests_cover_every_case():
    import json
    import os
    import scale_cases
    with open(os.path.join(os.path.dirname(__file__), "golden", "scale_digests.json")) as f:
        table = json.load(f)
    assert set(table) == set(scale_cases.CASES)
    for name, rec in table.items():
        assert rec["edges"] > 0 and len(rec["digest"]) == 32, name
