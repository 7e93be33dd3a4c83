"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Registers, winner rows, b0, calibrated cutoffs, top-N derived edge sets and
sComp are compared bit-exactly; edge weights exactly against the reference-
order oracle and within 1e-6 absolute of an FP64 recomputation.
"""
import numpy as np
import pytest

import oracle
from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-6   # edge weights vs the FP64 recomputation


def _concat(seqs):
    offs = np.zeros(len(seqs) + 1, np.int64)
    offs[1:] = np.cumsum([len(s) for s in seqs])
    return b"".join(seqs), offs


def _edge_cases():
    rng = np.random.default_rng(11)
    rnd = lambda n: bytes(rng.choice(list(b"ACGT"), size=n))
    return [
        b"",                          # empty contig
        b"ACG",                       # shorter than k
        b"ACGT",                      # exactly one k-mer (palindrome)
        b"NNNNNNNNNNNNNNNNNNNN",      # no valid base
        b"AAAAAAAAAAAAAAAAAAAAAAAAAAAAAAAA",   # homopolymer
        b"ACGT" * 100,                # palindromic 4-mers
        rnd(3000).lower(),            # lower case
        rnd(500) + b"N" + rnd(500) + b"NN" + rnd(3) + b"N" + rnd(700),  # N resets
        rnd(2501),
        bytes(rng.choice(list(b"ACGTNRYacgtn-"), size=4000)),         # IUPAC / gaps
        rnd(17) + b"X" * 5 + rnd(33),
    ]


@pytest.mark.parametrize("m", [2, 3, 17, 250, 500, 1000])
def test_winners_bit_exact(gpu_ctx, orc, m):
    asm = make_assembly(8, 150, 0, seed=100 + m, n_frac=0.01)
    seqs = _edge_cases() + asm.seqs
    buf, offs = _concat(seqs)
    p = api.default_params(m=m)
    got = gpu_ctx.build_pmh_winners(buf, offs, p)
    want = orc.build_winners(buf, offs, m=m)
    assert got.shape == want.shape
    bad = np.argwhere(got != want)
    assert bad.size == 0, f"{len(bad)} registers differ, first {bad[:5]}"


@pytest.mark.parametrize("k,gc", [(1, 1), (2, 1), (3, 1), (4, 0), (4, 1),
                                  (1, 2), (2, 2), (3, 2), (4, 2)])
def test_winners_k_and_gcnorm(gpu_ctx, orc, k, gc):
    asm = make_assembly(5, 80, 0, seed=7 * k + gc)
    buf, offs = _concat(_edge_cases() + asm.seqs)
    p = api.default_params(k=k, gc_norm=gc)
    got = gpu_ctx.build_pmh_winners(buf, offs, p)
    want = orc.build_winners(buf, offs, k=k, gc_norm=gc)
    assert np.array_equal(got, want)


def test_winners_against_reference(gpu_ctx, ref_lib):
    asm = make_assembly(10, 300, 0, seed=5, n_frac=0.01)
    buf, offs = _concat(_edge_cases() + asm.seqs)
    got = gpu_ctx.build_pmh_winners(buf, offs)
    assert np.array_equal(got, ref_lib.build_winners(buf, offs))


def test_pack_win16(gpu_ctx, orc):
    rng = np.random.default_rng(3)
    w = rng.integers(0, 2**32, size=100000, dtype=np.uint64).astype(np.uint32)
    w[:100] = 0
    w[100:200] = 0x00010001   # folds to 0 -> 1
    got = gpu_ctx.pack_win16(w)
    h = (w ^ (w >> 16)).astype(np.uint16)
    want = np.where(w == 0, 0, np.where(h == 0, 1, h)).astype(np.uint16)
    assert np.array_equal(got, want)


def _fp64_weights(asm, res, wc):
    """Edge weights recomputed in FP64 from the oracle's unit rows."""
    S = asm.n_samples
    if S <= 1:
        return None
    unit = res["unit"].astype(np.float64)
    d = asm.depth.astype(np.float64)
    cn = d.mean(axis=0)
    cn = np.where(cn > 1e-12, 1.0 / cn, 0.0)
    i, j = res["src"].astype(np.int64), res["dst"].astype(np.int64)
    rho = (unit[i] * unit[j]).sum(axis=1)
    x, y = d[i] * cn, d[j] * cn
    wj = np.minimum(x, y).sum(axis=1) / np.maximum(np.maximum(x, y).sum(axis=1), 1e-300)
    wj = np.clip(wj, 0, 1)
    dterm = np.minimum(np.maximum(rho, 0), wj)
    w = wc * res["scomp"].astype(np.float64) + (1 - wc) * dterm
    w[(rho < -0.3) | (w < 0.70)] = 0.0
    return w


def _graph_case(gpu_ctx, orc, G, N, S, seed, **kw):
    asm = make_assembly(G, N, S, seed=seed, absent_frac=0.1 if S > 2 else 0.0)
    buf, offs = asm.concat()
    w = orc.build_winners(buf, offs)
    op = oracle.default_params(asm.n, 500, S, **kw)
    want = orc.run_graph(op, w, asm.depth)
    gp = api.default_params(**kw)
    got = gpu_ctx.bin_graph(buf, offs, asm.depth, gp)
    assert got["b0"] == want["b0"]
    assert got["sim_cutoff"] == want["sim_cutoff"]
    ws, wd, wsc, wsw = oracle.sorted_edges(want)
    assert np.array_equal(got["src"], ws) and np.array_equal(got["dst"], wd), \
        f"edge sets differ: {len(got['src'])} vs {len(ws)}"
    assert np.array_equal(got["scomp"], wsc)
    assert np.array_equal(got["score"], wsw)
    fp = _fp64_weights(asm, dict(want, src=ws, dst=wd, scomp=wsc), 0.0 if S > 2 else 1.0)
    if fp is not None and S > 2:
        agree = (fp > 0) == (wsw > 0)
        err = np.abs(fp[agree] - wsw[agree].astype(np.float64))
        assert err.size == 0 or err.max() <= TOL_FP64
    return got


@pytest.mark.parametrize("S", [0, 1, 2, 5])
def test_graph_small_path(gpu_ctx, orc, S):
    g = _graph_case(gpu_ctx, orc, 20, 2000, S, seed=40 + S)
    assert g["path"] == 1


@pytest.mark.parametrize("S,extra", [(3, {}), (10, {}), (20, {}), (30, {}), (40, {}),
                                     (1, {}), (2, {}), (5, {"mutual": 0}),
                                     (20, {"win_bits": 32}), (10, {"abdfirst": 0})])
def test_graph_fused_path(gpu_ctx, orc, S, extra):
    g = _graph_case(gpu_ctx, orc, 30, 4000, S, seed=60 + S, force_path=2, **extra)
    assert g["path"] == 2


def test_build_graph_from_reference_winners(gpu_ctx, ref_lib):
    asm = make_assembly(20, 3000, 10, seed=9, absent_frac=0.1)
    buf, offs = asm.concat()
    w = ref_lib.build_winners(buf, offs)
    p = oracle.default_params(asm.n, 500, 10, force_path=2)
    want = ref_lib.run_graph(p, w, asm.depth)
    got = gpu_ctx.build_graph(w, asm.depth, api.default_params(force_path=2))
    ws, wd, wsc, wsw = oracle.sorted_edges(want)
    assert got["b0"] == want["b0"] and got["sim_cutoff"] == want["sim_cutoff"]
    assert np.array_equal(got["src"], ws) and np.array_equal(got["dst"], wd)
    assert np.array_equal(got["scomp"], wsc) and np.array_equal(got["score"], wsw)


def test_estimate_b0(gpu_ctx, ref_lib):
    asm = make_assembly(15, 1500, 0, seed=21)
    buf, offs = asm.concat()
    w = ref_lib.build_winners(buf, offs)
    p = oracle.default_params(asm.n, 500, 0)
    want = ref_lib.run_graph(p, w, np.zeros((asm.n, 0), np.float32))["b0"]
    w16 = gpu_ctx.pack_win16(w)
    assert gpu_ctx.estimate_pmh_baseline(w16) == want


def test_same_alone_and_repeated(gpu_ctx, orc):
    """Device buffers are reused across calls: results do not depend on history."""
    a = make_assembly(10, 800, 5, seed=31)
    b = make_assembly(12, 1200, 10, seed=32)
    ba, oa = a.concat()
    bb, ob = b.concat()
    first = gpu_ctx.bin_graph(ba, oa, a.depth)
    gpu_ctx.bin_graph(bb, ob, b.depth, api.default_params(force_path=2 if b.n > 2500 else 0))
    again = gpu_ctx.bin_graph(ba, oa, a.depth)
    for k in ("src", "dst", "scomp", "score"):
        assert np.array_equal(first[k], again[k])


def test_against_golden_fixtures(gpu_ctx):
    """Outputs of RabbitBin's own code, committed as fixtures (no reference tree
    is needed at run time)."""
    import os
    gdir = os.path.join(os.path.dirname(__file__), "golden")
    files = sorted(f for f in os.listdir(gdir) if f.endswith(".npz"))
    assert files
    for f in files:
        z = np.load(os.path.join(gdir, f))
        if "seqcat" not in z.files:
            continue                     # label fixtures (lpa.npz), checked in test_gpu_lpa.py
        seqcat, offs, m = z["seqcat"].tobytes(), z["offsets"], int(z["m"])
        w = gpu_ctx.build_pmh_winners(seqcat, offs, api.default_params(m=m))
        assert np.array_equal(w, z["winners32"]), f
        if "src" in z.files:
            p = api.default_params(m=m, force_path=int(z["force_path"]))
            g = gpu_ctx.bin_graph(seqcat, offs, z["depth"], p)
            assert g["b0"] == float(z["b0"]) and g["sim_cutoff"] == float(z["sim_cutoff"]), f
            assert np.array_equal(g["src"], z["src"]) and np.array_equal(g["dst"], z["dst"]), f
            assert np.array_equal(g["scomp"], z["scomp"]), f
            assert np.array_equal(g["score"], z["score"]), f


@pytest.mark.parametrize("N,S,fp", [(2599, 7, 2), (2601, 33, 2), (3001, 2, 2), (1999, 4, 1)])
def test_graph_ragged_sizes(gpu_ctx, orc, N, S, fp):
    """Row/column counts that leave partial CTA tiles."""
    _graph_case(gpu_ctx, orc, 25, N, S, seed=N, force_path=fp)


@pytest.mark.parametrize("kind", ["fractional", "wide_range"])
def test_graph_nonint_depths(gpu_ctx, orc, kind):
    """Coverage values that are not small integers: the column sums of the
    weighted-Jaccard norm must still round exactly as the sequential sum."""
    asm = make_assembly(20, 3000, 6, seed=77)
    rng = np.random.default_rng(5)
    d = asm.depth * rng.uniform(0.5, 1.5, size=asm.depth.shape).astype(np.float32)
    if kind == "wide_range":
        d[rng.random(d.shape) < 0.05] = np.float32(3e-30)
        d[rng.random(d.shape) < 0.01] *= np.float32(1e12)
    d = d.astype(np.float32)
    buf, offs = asm.concat()
    w = orc.build_winners(buf, offs)
    for fp in (1, 2):
        want = orc.run_graph(oracle.default_params(asm.n, 500, 6, force_path=fp), w, d)
        got = gpu_ctx.bin_graph(buf, offs, d, api.default_params(force_path=fp))
        s, dd, sc, sw = oracle.sorted_edges(want)
        assert got["sim_cutoff"] == want["sim_cutoff"]
        assert np.array_equal(got["src"], s) and np.array_equal(got["dst"], dd)
        assert np.array_equal(got["scomp"], sc) and np.array_equal(got["score"], sw)


@pytest.mark.parametrize("S,cap", [(3, None), (12, None), (20, None), (20, "4096")])
def test_streamed_pairs_equal_resident(S, cap):
    """rbg_bin_graph scores the pairs chunk by chunk behind the input copy with
    admission deferred until b0 is known (from S = 10 up), falling back to the
    whole pass when the stored survivors outgrow the list (forced here with a
    4096-pair first list, after which that S no longer streams); the graph
    equals the one of the resident path, which scores all pairs at once."""
    import os
    asm = make_assembly(30, 4000, S, seed=410 + S, absent_frac=0.1)
    buf, offs = asm.concat()
    assert len(buf) >= 8 * 16 * 65536          # eight input chunks
    p = api.default_params(force_path=2)
    if cap:
        os.environ["RBG_PAIR_CAP"] = cap
    try:
        ctx = api.Context(0)
        streamed = ctx.bin_graph(buf, offs, asm.depth, p)
        again = ctx.bin_graph(buf, offs, asm.depth, p)
    finally:
        os.environ.pop("RBG_PAIR_CAP", None)
    ctx.stage(buf, offs, asm.depth)
    ctx.run_resident(p)
    resident = ctx.fetch_graph()
    ctx.close()
    for got in (streamed, again):
        assert got["b0"] == resident["b0"] and got["sim_cutoff"] == resident["sim_cutoff"]
        for k in ("src", "dst", "scomp", "score"):
            assert np.array_equal(got[k], resident[k]), k


@pytest.mark.parametrize("S", [1, 5])
def test_graph_small_path_alu_compare(gpu_ctx, orc, S):
    """The dense regime on the integer-ALU register compare (RBG_DENSE_ALU=1)
    instead of the one-hot tensor-core kernel: the same graph."""
    import os
    os.environ["RBG_DENSE_ALU"] = "1"
    try:
        g = _graph_case(gpu_ctx, orc, 20, 1500, S, seed=70 + S)
    finally:
        os.environ.pop("RBG_DENSE_ALU", None)
    assert g["path"] == 1


@pytest.mark.parametrize("N,S", [(300, 5), (1000, 0), (5000, 3), (9000, 2)])
def test_graph_small_path_onehot_sizes(gpu_ctx, orc, N, S):
    """The one-hot tensor-core kernel at row/column counts that leave partial
    256-row and 256-column tiles, a single tile, and several column groups."""
    g = _graph_case(gpu_ctx, orc, max(4, N // 250), N, S, seed=900 + N)
    assert g["path"] == 1


@pytest.mark.parametrize("N,S", [(3000, 2), (6000, 5)])
def test_graph_small_path_onehot_cut(gpu_ctx, orc, N, S):
    """Candidate lists shorter than their column group (RBG_ONEHOT_CAP): the
    lists are cut to the K best inside the tensor-core kernel, several times
    per row, and the graph stays the same."""
    import os
    os.environ["RBG_ONEHOT_CAP"] = "1"          # the floor: K + 136 keys, rounded
    try:
        g = _graph_case(gpu_ctx, orc, 6, N, S, seed=950 + N)
    finally:
        os.environ.pop("RBG_ONEHOT_CAP", None)
    assert g["path"] == 1
