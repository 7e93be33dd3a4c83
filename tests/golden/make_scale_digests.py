"""Record RabbitBin's own graphs of the benchmark-scale parity cases.

    python tests/golden/make_scale_digests.py [case ...]

Runs in the build container, where the reference tree is present: the
reference harness (oracle/_ref) sketches each case of tests/scale_cases.py and
builds its graph with the reference's own graph code; the digest of the graph
sorted by (from, to) (edges, sComp, edge weights, b0, cutoff) is written to
scale_digests.json next to this script, with the edge count, b0 and cutoff.
The GPU tests compare the device graphs of the same seeded cases against these
digests (the GPU box has no reference tree).
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
import scale_cases  # noqa: E402

OUT = os.path.join(HERE, "scale_digests.json")


def main(names):
    ref = oracle.ref()
    if ref is None:
        raise SystemExit("reference tree not available")
    table = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            table = json.load(f)
    for name in names or list(scale_cases.CASES):
        t0 = time.time()
        asm, m, wb = scale_cases.assembly(name)
        buf, offs = asm.concat()
        w = ref.build_winners(buf, offs, m=m)
        p = oracle.default_params(asm.n, m, asm.n_samples, win_bits=wb)
        res = ref.run_graph(p, w, asm.depth)
        s, d, sc, sw = oracle.sorted_edges(res)
        g = dict(src=s, dst=d, scomp=sc, score=sw, b0=res["b0"], sim_cutoff=res["sim_cutoff"])
        table[name] = {"digest": scale_cases.digest(g), "n": asm.n, "S": asm.n_samples,
                       "m": m, "win_bits": wb, "edges": int(len(s)), "b0": res["b0"],
                       "sim_cutoff": res["sim_cutoff"]}
        print(name, table[name], f"{time.time() - t0:.1f} s", flush=True)
        with open(OUT, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
