"""Label propagation on the device (rbg_label_propagation*) against the
reference's own cluster_by_propagation (oracle/_ref) and the committed golden
labels: identical labels, both sweeps, every score rule, edge cases."""
import os
import subprocess
import sys

import numpy as np
import pytest

from rabbitbin_b200 import api
from test_lpa_cpu import _graph

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(autouse=True)
def _no_lpa_env(monkeypatch):
    monkeypatch.delenv("RABBIT_LPA_SCORE", raising=False)
    monkeypatch.delenv("RABBIT_PAR_LPA", raising=False)


@pytest.mark.parametrize("name", ["small_path_s5", "fused_s20_m64", "fused_s3_m96"])
@pytest.mark.parametrize("seed", [1, 7])
@pytest.mark.parametrize("sync", [False, True])
def test_labels_match_golden(gpu_ctx, name, seed, sync):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    L = np.load(os.path.join(GOLDEN, "lpa.npz"))
    n = len(g["offsets"]) - 1
    got, st = gpu_ctx.label_propagation(n, g["src"], g["dst"], g["score"], seed=seed,
                                        rule="fisher", synchronous=sync)
    want = L[f"{name}_{'sync' if sync else 'gs'}_{seed}"]
    assert (got == want).all(), int((got != want).sum())
    assert st["rounds"] >= 1 and st["arcs"] == 2 * int((g["score"] > 0).sum())


@pytest.mark.parametrize("seed", [0, 3])
@pytest.mark.parametrize("n,k,groups", [(3000, 40, 12), (6000, 24, 40)])
@pytest.mark.parametrize("sync", [False, True])
def test_random_graphs_match_reference(gpu_ctx, ref_lib, monkeypatch, seed, n, k, groups, sync):
    s, d, w = _graph(n, seed, k=k, groups=groups)
    if sync:
        monkeypatch.setenv("RABBIT_PAR_LPA", "1")
    want = ref_lib.label_propagation(n, s, d, w, seed=seed + 11)
    got, _ = gpu_ctx.label_propagation(n, s, d, w, seed=seed + 11, rule="fisher",
                                       synchronous=sync)
    assert (got == want).all(), int((got != want).sum())


def test_explicit_node_order(gpu_ctx, ref_lib):
    n = 2000
    s, d, w = _graph(n, 9, k=30, groups=6)
    order = np.random.default_rng(4).permutation(n).astype(np.uint32)
    want = ref_lib.label_propagation(n, s, d, w, node_order=order)
    got, _ = gpu_ctx.label_propagation(n, s, d, w, node_order=order, rule="fisher",
                                       synchronous=False)
    assert (got == want).all()


def test_high_degree_and_self_loops(gpu_ctx, ref_lib):
    # hubs above the shared table (384 arcs) and above the shared sort (4096 arcs),
    # a self-loop, isolated nodes
    rng = np.random.default_rng(5)
    n = 9000
    s, d, w = _graph(n, 2, k=8, groups=30)
    hub_a = np.full(5000, 1, np.uint32)
    hub_b = rng.choice(np.arange(2, n), 5000, replace=False).astype(np.uint32)
    hub2_b = rng.choice(np.arange(3, n), 600, replace=False).astype(np.uint32)
    src = np.concatenate([s, hub_a, np.full(600, 2, np.uint32), [5]]).astype(np.uint32)
    dst = np.concatenate([d, hub_b, hub2_b, [5]]).astype(np.uint32)
    sc = np.concatenate([w, rng.uniform(0.7, 0.99, 5600).astype(np.float32),
                         [np.float32(0.9)]]).astype(np.float32)
    want = ref_lib.label_propagation(n, src, dst, sc, seed=2)
    got, st = gpu_ctx.label_propagation(n, src, dst, sc, seed=2, rule="fisher",
                                        synchronous=False)
    assert (got == want).all(), int((got != want).sum())


_RULES_CHILD = r'''
import sys, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import oracle
from rabbitbin_b200 import api
from test_lpa_cpu import _graph
n = 3000
s, d, w = _graph(n, 8, k=30, groups=10)
want = oracle.ref().label_propagation(n, s, d, w, seed=5)
got, _ = api.Context(0).label_propagation(n, s, d, w, seed=5)   # rule and sweep from the env
sys.exit(0 if (got == want).all() else 1)
'''


@pytest.mark.parametrize("rule", ["tail", "logsum", "sum", "mean", "max"])
@pytest.mark.parametrize("sync", [False, True])
def test_score_rules_match_reference(ref_lib, rule, sync):
    env = dict(os.environ, RABBIT_LPA_SCORE=rule)
    if sync:
        env["RABBIT_PAR_LPA"] = "1"
    else:
        env.pop("RABBIT_PAR_LPA", None)
    r = subprocess.run([sys.executable, "-c", _RULES_CHILD, ROOT], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


def test_edge_cases(gpu_ctx):
    # no edges: every node keeps its label (the reference returns early)
    got, st = gpu_ctx.label_propagation(5, [], [], np.zeros(0, np.float32))
    assert (got == np.arange(5)).all() and st["rounds"] == 0
    # only zero scores: no incidence, one round without a change
    got, st = gpu_ctx.label_propagation(4, [0, 1], [1, 2], np.zeros(2, np.float32))
    assert (got == np.arange(4)).all() and st["arcs"] == 0
    # a pair joins; the later node in the order takes the other's label
    got, _ = gpu_ctx.label_propagation(3, [0], [1], np.array([0.9], np.float32),
                                       node_order=[1, 0, 2])
    assert got[0] == got[1] and got[2] == 2
    with pytest.raises(api.RbgError):
        gpu_ctx.label_propagation(3, [0], [1], np.array([-0.1], np.float32))
    with pytest.raises(api.RbgError):
        gpu_ctx.label_propagation(3, [0], [7], np.array([0.9], np.float32))
    with pytest.raises(api.RbgError):
        gpu_ctx.label_propagation(3, [0], [1], np.array([0.9], np.float32), node_order=[0, 0, 1])


def test_resident_graph(gpu_ctx, ref_lib):
    """On the graph rbg_bin_graph leaves on the device, as the serving path uses it."""
    g = np.load(os.path.join(GOLDEN, "fused_s3_m96.npz"))
    seqcat = g["seqcat"].tobytes()
    n = len(g["offsets"]) - 1
    p = api.default_params(m=int(g["m"]), force_path=2)
    res = gpu_ctx.bin_graph(seqcat, g["offsets"], g["depth"], p)
    got, st = gpu_ctx.label_propagation_resident(n, seed=1, rule="fisher", synchronous=False)
    want = ref_lib.label_propagation(n, res["src"], res["dst"], res["score"], seed=1)
    assert (got == want).all()
    L = np.load(os.path.join(GOLDEN, "lpa.npz"))
    assert (got == L["fused_s3_m96_gs_1"]).all()
