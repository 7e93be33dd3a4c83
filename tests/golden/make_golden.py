"""Regenerate the golden fixtures from RabbitBin's own code (oracle/_ref).

    python tests/golden/make_golden.py          # all fixtures
    python tests/golden/make_golden.py --lpa    # label-propagation labels only

Runs in the build container, where the reference tree is present: the
reference harness (src/probmh.cpp + the hot-path functions of
src/rabbitbin.cpp and src/impl/rb_graph.cpp, compiled in place) computes the
winner rows, b0, calibrated cutoff, edge set and edge weights of small seeded
assemblies; the outputs are stored as .npz next to this script.  The GPU box
has no reference tree, so the tests there compare against these files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rabbitbin_b200.synth import make_assembly  # noqa: E402

CASES = [
    # name, genomes, contigs, samples, seed, m, force_path, n_frac, absent, short
    ("small_path_s5", 8, 300, 5, 1, 500, 1, 0.01, 0.0, False),
    ("small_path_s1", 6, 200, 1, 2, 250, 1, 0.0, 0.0, False),
    ("fused_s20_m64", 12, 2600, 20, 3, 64, 2, 0.0, 0.1, True),
    ("fused_s3_m96", 10, 2600, 3, 4, 96, 2, 0.005, 0.1, True),
    ("sketch_only_m3", 3, 40, 0, 5, 3, 0, 0.05, 0.0, False),
]


def main():
    ref = oracle.ref()
    if ref is None:
        raise SystemExit("reference tree not available")
    for name, G, N, S, seed, m, fp, nf, ab, short in CASES:
        lens = dict(min_len=150, max_len=600, median_len=250.0) if short else {}
        asm = make_assembly(G, N, S, seed=seed, n_frac=nf, absent_frac=ab, **lens)
        seqs = [b"", b"ACG", b"ACGT" * 8, b"N" * 12] + asm.seqs
        offs = np.zeros(len(seqs) + 1, np.int64)
        offs[1:] = np.cumsum([len(s) for s in seqs])
        seqcat = b"".join(seqs)
        depth = np.concatenate([np.zeros((4, S), np.float32), asm.depth]) if S else \
            np.zeros((len(seqs), 0), np.float32)
        w = ref.build_winners(seqcat, offs, m=m)
        out = dict(seqcat=np.frombuffer(seqcat, np.uint8), offsets=offs, m=m,
                   winners32=w, S=S, force_path=fp, depth=depth)
        if fp:
            p = oracle.default_params(len(seqs), m, S, force_path=fp)
            res = ref.run_graph(p, w, depth)
            s, d, sc, sw = oracle.sorted_edges(res)
            out.update(src=s, dst=d, scomp=sc, score=sw, b0=res["b0"],
                       sim_cutoff=res["sim_cutoff"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, len(seqs), "contigs", len(out.get("src", [])), "edges")


LPA_GRAPHS = ["small_path_s5", "fused_s20_m64", "fused_s3_m96"]


def make_lpa():
    """Labels of the reference's label propagation (cluster_by_propagation,
    src/impl/rb_cluster.cpp:376-740) on the edge lists of the graph fixtures,
    sequential and synchronous sweeps, seeds 1 and 7 -> lpa.npz."""
    ref = oracle.ref()
    if ref is None:
        raise SystemExit("reference tree not available")
    out = {}
    for name in LPA_GRAPHS:
        g = np.load(os.path.join(HERE, name + ".npz"))
        n = len(g["offsets"]) - 1
        for seed in (1, 7):
            out[f"{name}_gs_{seed}"] = ref.label_propagation(n, g["src"], g["dst"], g["score"],
                                                             seed=seed)
            os.environ["RABBIT_PAR_LPA"] = "1"
            out[f"{name}_sync_{seed}"] = ref.label_propagation(n, g["src"], g["dst"],
                                                               g["score"], seed=seed)
            del os.environ["RABBIT_PAR_LPA"]
        out[f"{name}_order_1"] = ref.lpa_node_order(n, 1)
        print(name, n, "nodes", len(np.unique(out[f"{name}_gs_1"])), "labels")
    np.savez_compressed(os.path.join(HERE, "lpa.npz"), **out)


if __name__ == "__main__":
    if "--lpa" in sys.argv:
        make_lpa()
    else:
        main()
        make_lpa()
