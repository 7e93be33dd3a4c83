"""The one-permutation MinHash metric (RABBIT_PMH=0) on the device: bucket
values against the reference's own KmerSketch (src/rabbit_sketch.h) bit for
bit, and the graph with that metric (small path, and the large-N route with
its sampled calibration) against the reference's rb_cmd_bin sequence
(graph_sim -> jaccard_raw, no baseline) compiled in the harness: edges, sComp,
edge scores and the calibrated cutoff identical."""
import numpy as np
import pytest

import oracle
from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly

from test_oph_cpu import _fuzz

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,K,bits", [(500, 8, 2), (2, 1, 1), (64, 4, 1), (130, 15, 3),
                                      (1000, 21, 2), (4096, 12, 2), (250, 32, 7)])
def test_oph_signature_bit_exact(gpu_ctx, ref_lib, m, K, bits):
    cat, offs = _fuzz(m + K)
    p = api.default_params(m=m, oph_k=K, oph_bits=bits)
    got = gpu_ctx.build_oph_signature(cat, offs, p)
    want = ref_lib.oph_values(cat, offs, m, K, bits)
    assert np.array_equal(got, want)


def test_oph_signature_assembly(gpu_ctx, ref_lib):
    asm = make_assembly(10, 1500, 0, seed=77)
    buf, offs = asm.concat()
    p = api.default_params(m=500, oph_k=8, oph_bits=2)
    assert np.array_equal(gpu_ctx.build_oph_signature(buf, offs, p),
                          ref_lib.oph_values(buf, offs, 500, 8, 2))


def _oph_case(gpu_ctx, ref_lib, G, N, S, m, bits, seed, **kw):
    asm = make_assembly(G, N, S, seed=seed, absent_frac=0.1 if S > 2 else 0.0)
    buf, offs = asm.concat()
    op = oracle.default_params(asm.n, m, S, oph_k=8, oph_bits=bits, **kw)
    want = ref_lib.run_graph_oph(op, buf, offs, asm.depth)
    got = gpu_ctx.bin_graph(buf, offs, asm.depth,
                            api.default_params(m=m, oph_k=8, oph_bits=bits, **kw))
    assert got["path"] == 1 and got["b0"] == 0.0 == want["b0"]
    assert got["sim_cutoff"] == want["sim_cutoff"]
    ws, wd, wsc, wsw = oracle.sorted_edges(want)
    assert np.array_equal(got["src"], ws) and np.array_equal(got["dst"], wd), \
        f"edge sets differ: {len(got['src'])} vs {len(ws)}"
    assert np.array_equal(got["scomp"], wsc)
    assert np.array_equal(got["score"], wsw)
    assert len(ws) > 0
    return got


@pytest.mark.parametrize("S,m,bits", [(0, 500, 2), (1, 500, 2), (5, 500, 2), (10, 1000, 1),
                                      (5, 250, 3)])
def test_oph_graph_small_path(gpu_ctx, ref_lib, S, m, bits):
    _oph_case(gpu_ctx, ref_lib, 20, 2000, S, m, bits, seed=90 + S)


@pytest.mark.parametrize("S", [0, 5, 20])
def test_oph_graph_large_route(gpu_ctx, ref_lib, S):
    """N > 25000 route of the metric (forced at 4000 contigs): the cutoff from
    ten 2500-contig samples, then the small path's all-pairs graph."""
    g = _oph_case(gpu_ctx, ref_lib, 30, 4000, S, 500, 2, seed=120 + S, force_path=2)
    assert g["path"] == 1


def test_oph_and_index_assemblies_in_a_batch(gpu_ctx):
    """The batch form takes assemblies on the one-permutation metric and the
    inverted-index graph beside ProbMinHash ones: they run through the
    single-assembly path inside the same call, each graph identical to
    rbg_bin_graph's on that assembly alone."""
    ent = []
    for seed, (G, N, S), kw in ((5, (10, 3000, 5), dict(oph_k=8)), (6, (8, 2000, 3), {}),
                                (7, (6, 1500, 2), dict(graph_index=1)),
                                (8, (9, 2600, 4), dict(oph_k=6))):
        asm = make_assembly(G, N, S, seed=seed)
        buf, offs = asm.concat()
        ent.append((buf, offs, asm.depth, api.default_params(**kw)))
    got, st = gpu_ctx.bin_batch(ent)
    assert st["n_assemblies"] == 1                         # the ProbMinHash one
    for g, e in zip(got, ent):
        want = gpu_ctx.bin_graph(*e)
        for k in ("src", "dst", "scomp", "score"):
            assert np.array_equal(np.asarray(g[k]), np.asarray(want[k])), k
    with pytest.raises(api.RbgError):                      # winner rows are ProbMinHash
        gpu_ctx.build_pmh_winners(ent[0][0], ent[0][1], api.default_params(oph_k=8))
