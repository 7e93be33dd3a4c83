"""The benchmark-scale parity cases: seeded assemblies with the shapes of the
benchmark configurations, shared by the GPU parity tests and the script that
records the reference harness's graphs of them (tests/golden/make_scale_digests.py).

* config0_w16 / config0_w32: 20 genomes, 2,000 large + 500 short contigs, S = 5,
  m = 500, K = 200 (the reference's N <= 25000 path, calibrate_sim_cutoff +
  build_graph_allpairs, src/impl/rb_graph.cpp:1362-1384, :7-72), with the
  default 16-bit winners and with RABBIT_WIN_BITS=32;
* config1: 100 genomes, 50,000 contigs, S = 20 (gen_fused_calib_graph,
  src/impl/rb_graph.cpp:501-1356, mutual filter and abundance prune on);
* batch_n88584: the largest assembly of the 64-assembly mixed stream (seed 2):
  88,584 contigs, S = 5, m = 500 (weak-prune regime of the fused path);
* config3: 300 genomes, 300,000 contigs, S = 30 with 10% of genomes absent per
  sample (4.5e10 pairs through the fused path).
"""
import hashlib

import numpy as np

CASES = {
    "config0_w16": dict(genomes=20, contigs=2000, small=500, S=5, seed=0, m=500, win_bits=16),
    "config0_w32": dict(genomes=20, contigs=2000, small=500, S=5, seed=0, m=500, win_bits=32),
    "config1": dict(genomes=100, contigs=50000, S=20, seed=1, m=500, win_bits=16),
    "batch_n88584": dict(stream_seed=2, stream_count=64, stream_index=55, m=500, win_bits=16),
    "config3": dict(genomes=300, contigs=300000, S=30, seed=3, absent=0.1, m=500, win_bits=16),
}


def assembly(name):
    """(Assembly, m, win_bits) of one case."""
    from rabbitbin_b200.synth import make_assembly
    c = CASES[name]
    if "stream_seed" in c:
        from rabbitbin_b200.workloads import draw_sizes
        n, S, m = draw_sizes(c["stream_count"], c["stream_seed"], 1000, 100000,
                             (3, 5, 10, 30), (250, 500, 1000))[c["stream_index"]]
        assert m == c["m"]
        g = int(min(300, max(10, n // 500)))
        seed = c["stream_seed"] * 100003 + c["stream_index"]
        return make_assembly(g, n, S, seed=seed), m, c["win_bits"]
    asm = make_assembly(c["genomes"], c["contigs"], c["S"], seed=c["seed"],
                        n_small=c.get("small", 0), absent_frac=c.get("absent", 0.0))
    return asm, c["m"], c["win_bits"]


def digest(g):
    """Digest of a graph sorted by (from, to): edges, sComp, weights, b0, cutoff."""
    h = hashlib.blake2b(digest_size=16)
    for k in ("src", "dst", "scomp", "score"):
        h.update(np.ascontiguousarray(g[k]).tobytes())
    h.update(np.float64([g["b0"], g["sim_cutoff"]]).tobytes())
    return h.hexdigest()
