"""GPU parity at the benchmark configurations.

The device graph of each case of scale_cases.py (the benchmark shapes: the
2,000-contig small path at 16- and 32-bit winners, the 50,000-contig binning
assembly, the largest assembly of the mixed batch stream run through
rbg_bin_batch, the 300,000-contig assembly) is compared with RabbitBin's own
code: against the digest the reference harness recorded for the same seeded
inputs (tests/golden/scale_digests.json, made by make_scale_digests.py), and,
where the harness is present and quick (N <= 50,000), against a live run of
it.  Edges, sComp, edge weights, b0 and the cutoff must be bit-identical.  The
edge weights' distance to the FP64 recomputation (oracle.fp64_edge_weights)
must stay within 1e-6 and is reported in the session summary.
"""
import json
import os

import numpy as np
import pytest

import oracle
import scale_cases
from rabbitbin_b200 import api

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-6
HERE = os.path.dirname(os.path.abspath(__file__))

with open(os.path.join(HERE, "golden", "scale_digests.json")) as _f:
    DIGESTS = json.load(_f)


def _sorted(g):
    order = np.lexsort((g["dst"], g["src"]))
    return {k: np.asarray(g[k])[order] for k in ("src", "dst", "scomp", "score")} | \
        {"b0": g["b0"], "sim_cutoff": g["sim_cutoff"]}


def _check(name, g, asm, fp64_report, live=None):
    want = DIGESTS[name]
    assert g["b0"] == want["b0"], f"{name}: b0 {g['b0']} vs {want['b0']}"
    assert g["sim_cutoff"] == want["sim_cutoff"], f"{name}: cutoff"
    assert len(g["src"]) == want["edges"], f"{name}: {len(g['src'])} edges vs {want['edges']}"
    assert scale_cases.digest(_sorted(g)) == want["digest"], f"{name}: graph digest differs"
    if live is not None:
        s, d, sc, sw = oracle.sorted_edges(live)
        gs = _sorted(g)
        assert np.array_equal(gs["src"], s) and np.array_equal(gs["dst"], d)
        assert np.array_equal(gs["scomp"], sc) and np.array_equal(gs["score"], sw)
    rep = oracle.fp64_report(asm.depth, g)
    fp64_report[name] = rep
    assert rep["max_abs_err_fp64"] <= TOL_FP64, f"{name}: {rep}"
    assert rep["max_margin_disagreeing"] <= TOL_FP64, f"{name}: {rep}"


@pytest.mark.parametrize("name", ["config0_w16", "config0_w32", "config1", "config3"])
def test_benchmark_config_graph(gpu_ctx, fp64_report, name):
    asm, m, wb = scale_cases.assembly(name)
    buf, offs = asm.concat()
    g = gpu_ctx.bin_graph(buf, offs, asm.depth, api.default_params(m=m, win_bits=wb))
    assert g["path"] == (1 if asm.n <= 25000 else 2)
    live = None
    ref = oracle.ref()
    if ref is not None and asm.n <= 50000:
        w = ref.build_winners(buf, offs, m=m)
        live = ref.run_graph(oracle.default_params(asm.n, m, asm.n_samples, win_bits=wb),
                             w, asm.depth)
    _check(name, g, asm, fp64_report, live)


def test_batch_stream_largest_assembly(gpu_ctx, fp64_report):
    """The 88,584-contig assembly of the mixed stream, batched with three other
    assemblies of the stream (other S and m) in one rbg_bin_batch call: its
    graph is the reference's, the others equal rbg_bin_graph alone."""
    from rabbitbin_b200.workloads import iter_stream
    big, m, wb = scale_cases.assembly("batch_n88584")
    others = [it for _, it in zip(range(3), iter_stream(3, seed=2))]
    ent = []
    for it in others:
        b, o = it.asm.concat()
        ent.append((b, o, it.asm.depth, api.default_params(m=it.m)))
    bb, bo = big.concat()
    ent.insert(1, (bb, bo, big.depth, api.default_params(m=m, win_bits=wb)))
    got, st = gpu_ctx.bin_batch(ent)
    _check("batch_n88584", got[1], big, fp64_report)
    for k in (0, 2, 3):
        alone = gpu_ctx.bin_graph(*ent[k])
        assert scale_cases.digest(_sorted(got[k])) == scale_cases.digest(_sorted(alone))
