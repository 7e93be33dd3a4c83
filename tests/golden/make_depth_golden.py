"""Regenerate tests/golden/depth.npz from RabbitBin's own depth code.

    python tests/golden/make_depth_golden.py

Runs in the build container, where the reference tree is present: the
reference's depth_accumulate_sample (src/rabbit_depth.cpp:1615-1685, with
caldepth, ReadStatistics and CheckRead, compiled by oracle/build.py into
oracle/_ref/librbref_depth.so) sums the seeded BAMs of tests/depth_cases.py
under every parameter set there.  The stored sums and read lengths let the
tests check the library where that harness is absent.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from depth_cases import CASES, PARAMS, case  # noqa: E402
from rabbitbin_b200.synth import bam_records  # noqa: E402


def main():
    if oracle.ref_depth() is None:
        raise SystemExit("reference tree not available")
    out = {}
    for name in CASES:
        _, _, bam = case(name)
        recs, tl, _ = bam_records(bam)
        for i, (pid, edge, inc, mq, dq) in enumerate(PARAMS):
            s, avg = oracle.depth_accumulate_ref(recs, tl, pid, edge, inc, mq)
            out[f"{name}/{i}/sums"] = s
            out[f"{name}/{i}/avg"] = np.int32(avg)
            if dq:
                su, _ = oracle.depth_accumulate_ref(recs, tl, pid, edge, inc, max(mq, dq))
                out[f"{name}/{i}/sums_u"] = su
    np.savez_compressed(os.path.join(HERE, "depth.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
