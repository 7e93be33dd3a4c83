"""Batch form (rbg_bin_batch): each assembly's graph equals the single-assembly
call on that assembly alone, bit for bit, whatever else is in the batch.

The single-assembly path is itself checked against the oracle and the
reference (test_gpu_parity.py); here the mix covers every all-pairs variant
(dense, tensor-core KS = 1, 2, 4), both calibration paths, three sketch sizes,
two k values (two count groups), and empty and tiny assemblies.
"""
import os

import numpy as np
import pytest

from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly

pytestmark = pytest.mark.gpu

KEYS = ("src", "dst", "scomp", "score")


def _mix():
    """(assembly, params kwargs) covering the batch engine's groupings."""
    cases = [
        ((8, 700, 3, 1), dict(m=250)),                       # small path
        ((10, 1500, 5, 2), dict(m=500)),                     # small path
        ((12, 3200, 10, 3), dict(m=1000, force_path=2)),     # fused, tensor cores KS=1
        ((12, 2600, 30, 4), dict(m=500, force_path=2)),      # fused, KS=2
        ((6, 2700, 40, 5), dict(m=500, force_path=2)),       # fused, KS=4
        ((5, 400, 0, 6), dict(m=500)),                       # no depth file
        ((5, 300, 1, 7), dict(m=250)),                       # S = 1
        ((5, 350, 2, 8), dict(m=500)),                       # S = 2 (w_comp = 1)
        ((10, 2800, 20, 9), dict(m=500, force_path=2, mutual=0)),
        ((10, 2800, 20, 10), dict(m=500, force_path=2, win_bits=32)),
        ((10, 2900, 10, 11), dict(m=500, force_path=2, abdfirst=0)),   # fused, dense
        ((6, 900, 5, 12), dict(m=500, max_edges=100)),
        ((6, 800, 5, 13), dict(m=500, k=3)),                 # another count group
    ]
    out = []
    for (g, n, s, seed), kw in cases:
        a = make_assembly(g, n, s, seed=700 + seed, absent_frac=0.1 if s > 2 else 0.0)
        out.append((a, kw))
    return out


@pytest.fixture(scope="module")
def mix():
    return _mix()


def _entries(mix, extra=()):
    ent = []
    for a, kw in mix:
        buf, offs = a.concat()
        ent.append((buf, offs, a.depth, api.default_params(**kw)))
    rng = np.random.default_rng(5)
    tiny = [bytes(rng.choice(list(b"ACGT"), size=3000)) for _ in range(3)]
    offs = np.array([0, 3000, 6000, 9000], np.int64)
    ent.append((b"".join(tiny), offs, np.ones((3, 4), np.float32), api.default_params()))
    ent.append((b"", np.zeros(1, np.int64), np.zeros((0, 5), np.float32), api.default_params()))
    return ent + list(extra)


def _alone(ctx, ent):
    out = []
    for buf, offs, depth, p in ent:
        if len(offs) == 1:
            out.append(None)
            continue
        out.append(ctx.bin_graph(buf, offs, depth, p))
    return out


def _same(got, want, i):
    if want is None:
        assert len(got["src"]) == 0, i
        return
    assert got["path"] == want["path"], i
    assert got["b0"] == want["b0"] and got["sim_cutoff"] == want["sim_cutoff"], i
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), (i, k)


def test_batch_equals_alone(gpu_ctx, mix):
    ent = _entries(mix)
    want = _alone(gpu_ctx, ent)
    got, st = gpu_ctx.bin_batch(ent)
    assert st["n_assemblies"] == len(ent)
    assert st["rows"] == sum(len(e[1]) - 1 for e in ent)
    for i, (g, w) in enumerate(zip(got, want)):
        _same(g, w, i)
    assert st["edges"] == sum(len(g["src"]) for g in got)
    # a second call reuses (updates) the captured graphs
    again, st2 = gpu_ctx.bin_batch(ent)
    for i, (g, w) in enumerate(zip(again, want)):
        _same(g, w, i)
    assert st2["graph_launches"] == 3
    # a call's graphs share one pinned block: graphs kept while the others are
    # freed stay intact through later calls
    keep = {i: again[i] for i in range(0, len(again), 2)}
    del again, got
    third, _ = gpu_ctx.bin_batch(ent)
    fourth, _ = gpu_ctx.bin_batch(ent)
    for i, g in keep.items():
        _same(g, want[i], i)
    for i, (g, w) in enumerate(zip(third, want)):
        _same(g, w, i)
    del third
    for i, (g, w) in enumerate(zip(fourth, want)):
        _same(g, w, i)


def test_batch_order_and_subsets(gpu_ctx, mix):
    """Results do not depend on an assembly's position or its neighbours."""
    ent = _entries(mix)
    want = _alone(gpu_ctx, ent)
    perm = np.random.default_rng(1).permutation(len(ent))
    got, _ = gpu_ctx.bin_batch([ent[i] for i in perm])
    for j, i in enumerate(perm):
        _same(got[j], want[i], int(i))
    sub = [0, 4, 11]
    got, _ = gpu_ctx.bin_batch([ent[i] for i in sub])
    for j, i in enumerate(sub):
        _same(got[j], want[i], i)


def test_batch_without_graphs(gpu_ctx, mix):
    ent = _entries(mix)[:6]
    want = _alone(gpu_ctx, ent)
    os.environ["RBG_NO_GRAPHS"] = "1"
    try:
        got, st = gpu_ctx.bin_batch(ent)
    finally:
        del os.environ["RBG_NO_GRAPHS"]
    assert st["graph_launches"] == 0
    for i, (g, w) in enumerate(zip(got, want)):
        _same(g, w, i)


def test_batch_empty_and_errors(gpu_ctx, mix):
    got, st = gpu_ctx.bin_batch([])
    assert got == [] and st["n_assemblies"] == 0
    a, _ = mix[0]
    buf, offs = a.concat()
    with pytest.raises(api.RbgError) as e:
        gpu_ctx.bin_batch([(buf, offs, a.depth, api.default_params(m=1))])
    assert e.value.code == -1
    with pytest.raises(api.RbgError):                    # fused path needs n > 2500
        gpu_ctx.bin_batch([(buf, offs, a.depth, api.default_params(force_path=2))])
    # the context stays usable after a rejected call
    got, _ = gpu_ctx.bin_batch([(buf, offs, a.depth, api.default_params(m=250))])
    _same(got[0], gpu_ctx.bin_graph(buf, offs, a.depth, api.default_params(m=250)), 0)


def test_autotuner_keeps_results(tmp_path):
    """The autotuner times three all-pairs tile shapes on the first batch that
    meets a (variant, m, log2 n) key and keeps the fastest; the graphs equal
    the fixed rule's (RBG_NO_AUTOTUNE), and a second call meets no new key."""
    import os
    asms = []
    for i, (n, s) in enumerate([(3000, 20), (26000, 20), (1500, 5), (27000, 5)]):
        a = make_assembly(max(5, n // 300), n, s, seed=960 + i, absent_frac=0.1)
        buf, offs = a.concat()
        asms.append((buf, offs, a.depth))
    tuned = api.Context(0)
    first, st1 = tuned.bin_batch(asms)
    again, st2 = tuned.bin_batch(asms)
    assert st1["tuned_keys"] > 0 and st2["tuned_keys"] == 0
    os.environ["RBG_NO_AUTOTUNE"] = "1"
    try:
        fixed = api.Context(0)
        want, st3 = fixed.bin_batch(asms)
        assert st3["tuned_keys"] == 0
    finally:
        del os.environ["RBG_NO_AUTOTUNE"]
    for g1, g2, w in zip(first, again, want):
        for k in ("src", "dst", "scomp", "score"):
            assert np.array_equal(g1[k], w[k]) and np.array_equal(g2[k], w[k])
    tuned.close()
    fixed.close()


def test_batch_pair_list_overflow(mix):
    """A first pair list too small for the symmetric pass: the call runs the
    graph stage again, resident, with a larger list; graphs unchanged."""
    ent = _entries(mix)
    ref = api.Context(0)
    want = _alone(ref, ent)
    ref.close()
    os.environ["RBG_PAIR_CAP"] = "2048"
    try:
        small = api.Context(0)
        got, _ = small.bin_batch(ent)
        again, _ = small.bin_batch(ent)
    finally:
        del os.environ["RBG_PAIR_CAP"]
    for i, (g, w) in enumerate(zip(got, want)):
        _same(g, w, i)
    for i, (g, w) in enumerate(zip(again, want)):
        _same(g, w, i)
    small.close()
