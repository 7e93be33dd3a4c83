"""Seeded BAM cases of the depth summariser's tests (shared by the CPU and GPU
tests and by tests/golden/make_depth_golden.py)."""
import numpy as np

from rabbitbin_b200.synth import BAM_CLEAN, make_bam

# name: (contig lengths, depth seed, BAM options)
_LENS = np.array([5000, 200, 80000, 1000, 0, 150, 3000, 400, 151, 152, 1, 2, 3, 12000],
                 dtype=np.uint32)

CASES = {
    "edge_mix": (np.tile(_LENS, 12), 1, dict(seed=11)),
    "edge_mix_straddle": (np.tile(_LENS, 12), 2, dict(seed=12, straddle=True)),
    "short_reads": (np.tile(_LENS, 8), 3, dict(seed=13, read_len=60)),
    "long_reads": (np.tile(_LENS, 8), 4, dict(seed=14, read_len=700, p_indel=0.4)),
    "clean": (np.tile(_LENS, 6), 5, dict(seed=15, **BAM_CLEAN)),
    "all_overhang": (np.array([500, 800, 1200, 300] * 10, np.uint32), 6,
                     dict(seed=16, p_overhang=0.6, p_soft=0.4)),
    "few_reads": (np.array([300, 400], np.uint32), 7, dict(seed=17, n_unmapped_tail=3)),
}

# depth parameters: (percent identity, max edge, include edges, min MAPQ, dual MAPQ)
PARAMS = [
    (0.97, 75, False, 0, 0),
    (0.90, 75, False, 20, 30),
    (0.50, 0, False, 0, 0),
    (0.97, 200, True, 0, 0),
    (0.97, 10, False, 5, 0),
]


def case(name, depth_scale=1.0):
    lens, dseed, opts = CASES[name]
    depth = np.random.default_rng(dseed).uniform(0.2, 25.0, len(lens)) * depth_scale
    return lens, depth, make_bam(lens, depth, **opts)
