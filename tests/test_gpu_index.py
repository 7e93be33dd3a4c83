"""RABBIT_GRAPH_INDEX=1 on the device against RabbitBin's own
build_similarity_graph (src/impl/rb_graph.cpp:199-383) with its inverted
index (src/rabbit_invidx.h:51-160) built by one thread.

The index restricts each row's neighbours to contigs sharing at least
minCommon one-permutation sketch keys; candidates are taken in the order the
posting-list walk first meets them and kept by a max-edges heap whose strict
insertion rule makes ties at the boundary depend on that order, so small
max-edges values are part of the cases.  Edges, sComp and weights must be
identical.  (With several insertion threads the reference's own posting-list
order, and with it the tie-breaking, varies from run to run; one thread fixes
it in contig order, the order used here.)
"""
import numpy as np
import pytest

import oracle
from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,S,mc,K", [(2000, 5, 0, 200), (2000, 5, 80, 200), (2000, 5, 120, 200),
                                      (2000, 5, 150, 200), (1500, 1, 100, 5), (900, 0, 60, 3),
                                      (2600, 10, 40, 20)])
def test_index_graph_against_reference(gpu_ctx, ref_lib, N, S, mc, K):
    asm = make_assembly(max(6, N // 100), N, S, seed=500 + N + mc, absent_frac=0.1 if S > 2 else 0.0)
    buf, offs = asm.concat()
    w = ref_lib.build_winners(buf, offs)
    rp = oracle.default_params(asm.n, 500, S, max_edges=K, graph_index=1, min_common=mc)
    want = ref_lib.run_graph_index(rp, buf, offs, w, asm.depth)
    gp = api.default_params(max_edges=K, graph_index=1, min_common=mc)
    got = gpu_ctx.bin_graph(buf, offs, asm.depth, gp)
    assert got["path"] == 1
    assert got["b0"] == want["b0"] and got["sim_cutoff"] == want["sim_cutoff"]
    s, d, sc, sw = oracle.sorted_edges(want)
    assert np.array_equal(got["src"], s) and np.array_equal(got["dst"], d), \
        f"edge sets differ: {len(got['src'])} vs {len(s)}"
    assert np.array_equal(got["scomp"], sc) and np.array_equal(got["score"], sw)


def test_index_graph_through_batch(gpu_ctx):
    """The batch call runs an index-graph assembly through the single-assembly
    path: the same graph as rbg_bin_graph."""
    asm = make_assembly(5, 300, 3, seed=7)
    buf, offs = asm.concat()
    e = (buf, offs, asm.depth, api.default_params(graph_index=1))
    got, _ = gpu_ctx.bin_batch([e])
    want = gpu_ctx.bin_graph(*e)
    for k in ("src", "dst", "scomp", "score"):
        assert np.array_equal(np.asarray(got[0][k]), np.asarray(want[k])), k
