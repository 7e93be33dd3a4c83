"""Seeded mixed-size assembly streams for the batching and serving forms.

A stream is a list of independent assemblies whose contig counts are
log-uniform in [n_min, n_max], with S drawn from a set of sample counts and
the sketch size m from a set of register counts; contig lengths follow the
single-assembly law (log-normal, median 6 kb, sigma 0.8, clipped to
[2500, 80000]) and depths the lognormal genome x sample law of synth.py.
Genomes per assembly: one per 500 contigs, between 10 and 300 (the
binning-scale assembly has 100 genomes for 50,000 contigs).
"""
from dataclasses import dataclass
from typing import Iterator, List, Sequence

import numpy as np

from .synth import Assembly, make_assembly


@dataclass
class StreamItem:
    asm: Assembly
    S: int
    m: int
    seed: int

    @property
    def n(self) -> int:
        return self.asm.n


def draw_sizes(count: int, seed: int, n_min: int, n_max: int,
               s_choices: Sequence[int], m_choices: Sequence[int]):
    """(n, S, m) of each assembly of the stream."""
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=count)).round().astype(np.int64)
    S = rng.choice(np.asarray(s_choices), size=count)
    m = rng.choice(np.asarray(m_choices), size=count)
    return [(int(a), int(b), int(c)) for a, b, c in zip(n, S, m)]


def iter_stream(count: int, seed: int, n_min: int = 1000, n_max: int = 100000,
                s_choices: Sequence[int] = (3, 5, 10, 30),
                m_choices: Sequence[int] = (250, 500, 1000)) -> Iterator[StreamItem]:
    """The assemblies of one mixed stream, generated one at a time (the
    batching form's batch: 64 assemblies, n in [1e3, 1e5], S in {3, 5, 10, 30},
    m in {250, 500, 1000})."""
    for i, (n, S, m) in enumerate(draw_sizes(count, seed, n_min, n_max, s_choices, m_choices)):
        g = int(min(300, max(10, n // 500)))
        s = seed * 100003 + i
        yield StreamItem(make_assembly(g, n, S, seed=s), S, m, s)


def mixed_stream(count: int, seed: int, **kw) -> List[StreamItem]:
    return list(iter_stream(count, seed, **kw))
