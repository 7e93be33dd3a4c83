"""Seeded synthetic metagenome assemblies (contigs + MetaBAT-layout depth).

The reference names no public dataset for its graph-construction path, so every
workload here is generated from a fixed seed with the shapes and value laws of
the benchmark configurations:

* genomes: order-3 DNA Markov chains, 64 contexts x Dirichlet(0.5) transition
  rows, GC content tilted into U[0.30, 0.70] (exponential tilt of the G/C
  transition probabilities, bisection on the chain's stationary GC);
* contigs: cut without overlap from their genome, random strand, lengths
  log-normal (median 6 kb, sigma 0.8) clipped to [2500, 80000] (large contigs,
  the ones the graph is built on) plus optional short contigs of 1000-2499 bp;
* depth: per genome x sample mean ~ lognormal(mu=2, sigma=1), contig mean =
  Poisson(genome mean) stored as float32 (ties at low depth are intended), an
  optional fraction of genomes absent (depth 0) per sample; variance = mean.

Each contig is an independent chain drawn by a small C generator
(csrc/synth_chain.c, splitmix64 streams seeded from numpy), so a 400 Mbp
assembly takes about a second.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np



@dataclass
class Assembly:
    """Large contigs of one assembly plus their coverage table."""
    seqs: List[bytes]                 # ASCII, FASTA order
    depth: np.ndarray                 # float32 [n, S] contig mean depth per sample
    genome_of: np.ndarray             # int32 [n] source genome (for diagnostics)
    small_seqs: List[bytes] = field(default_factory=list)
    names: Optional[List[str]] = None

    @property
    def n(self) -> int:
        return len(self.seqs)

    @property
    def n_samples(self) -> int:
        return int(self.depth.shape[1]) if self.depth.ndim == 2 else 0

    def concat(self):
        """(bytes buffer, int64 offsets[n+1]) of the large contigs."""
        lens = np.fromiter((len(s) for s in self.seqs), dtype=np.int64, count=self.n)
        offs = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(lens, out=offs[1:])
        return b"".join(self.seqs), offs


def _stationary(P):
    """Stationary distribution of the 64-context chain with rows P[ctx, b]."""
    T = np.zeros((64, 64))
    c = np.repeat(np.arange(64), 4)
    np.add.at(T, (c, ((c << 2) | np.tile(np.arange(4), 64)) & 63), P.reshape(-1))
    # pi (T - I) = 0 with sum(pi) = 1: one equation replaced by the normalisation
    A = (T - np.eye(64)).T
    A[-1, :] = 1.0
    rhs = np.zeros(64)
    rhs[-1] = 1.0
    pi = np.linalg.solve(A, rhs)
    return pi / pi.sum()


def _gc_of(P):
    pi = _stationary(P)
    return float((pi[:, None] * P)[:, 1:3].sum())


def _tilted(P0, theta):
    w = P0 * np.exp(theta * np.array([0.0, 1.0, 1.0, 0.0]))
    return w / w.sum(axis=1, keepdims=True)


def _genome_tables(rng, n_genomes):
    tabs = np.zeros((n_genomes, 64, 4))
    for g in range(n_genomes):
        P0 = rng.dirichlet(np.full(4, 0.5), size=64)
        P0 = np.maximum(P0, 1e-6)
        P0 /= P0.sum(axis=1, keepdims=True)
        target = rng.uniform(0.30, 0.70)
        lo, hi = -12.0, 12.0
        for _ in range(40):
            mid = 0.5 * (lo + hi)
            if _gc_of(_tilted(P0, mid)) < target:
                lo = mid
            else:
                hi = mid
        tabs[g] = _tilted(P0, 0.5 * (lo + hi))
    return tabs


_chain_lib = None


def _chain_so():
    """The small C generator (built next to this file by rabbitbin_b200.build)."""
    global _chain_lib
    if _chain_lib is None:
        import ctypes
        import os
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsynth_chain.so")
        if not os.path.exists(path):
            from . import build as _b
            _b.build_synth()
        _chain_lib = ctypes.CDLL(path)
    return _chain_lib


def _chains(rng, tabs, genome_ids, lengths):
    """ASCII bases of one independent chain per (genome id, length) request."""
    import ctypes
    n = len(lengths)
    offs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.asarray(lengths, dtype=np.int64), out=offs[1:])
    cum = np.ascontiguousarray(np.cumsum(tabs, axis=2)[:, :, :3], dtype=np.float64)
    gid = np.ascontiguousarray(genome_ids, dtype=np.int32)
    seeds = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
    # filled here, on one thread: the generator's threads would otherwise take
    # the first-touch page faults of the whole buffer concurrently (slow)
    out = np.empty(int(offs[-1]), dtype=np.uint8)
    out.fill(0)
    P = ctypes.c_void_p
    _chain_so().synth_chains(P(cum.ctypes.data), P(gid.ctypes.data), P(offs.ctypes.data),
                             P(seeds.ctypes.data), ctypes.c_int64(n), P(out.ctypes.data))
    return out, offs


def _lognormal_lengths(rng, n, lo, hi, median=6000.0, sigma=0.8):
    L = np.exp(rng.normal(np.log(median), sigma, size=n))
    return np.clip(L, lo, hi).astype(np.int64)


def make_assembly(n_genomes: int, n_contigs: int, n_samples: int, seed: int,
                  n_small: int = 0, absent_frac: float = 0.0,
                  min_len: int = 2500, max_len: int = 80000,
                  median_len: float = 6000.0, n_frac: float = 0.0) -> Assembly:
    """One synthetic assembly.  ``n_frac`` sprinkles N runs into contigs (edge
    cases for the k-mer reset logic)."""
    rng = np.random.default_rng(seed)
    tabs = _genome_tables(rng, n_genomes)
    genome_of = rng.integers(0, n_genomes, size=n_contigs).astype(np.int32)
    lengths = _lognormal_lengths(rng, n_contigs, min_len, max_len, median_len)
    small_g = rng.integers(0, n_genomes, size=n_small).astype(np.int32)
    small_len = rng.integers(1000, 2500, size=n_small).astype(np.int64)
    allbuf, offs = _chains(rng, tabs, np.concatenate([genome_of, small_g]),
                           np.concatenate([lengths, small_len]))
    flip = rng.random(len(offs) - 1) < 0.5          # random strand
    comp = np.zeros(256, dtype=np.uint8)
    comp[list(b"ACGT")] = list(b"TGCA")
    seqs = []
    for k in range(len(offs) - 1):
        a = allbuf[offs[k]:offs[k + 1]]
        if flip[k]:
            a = comp[a[::-1]]
        if n_frac > 0.0 and len(a) > 0:
            a = a.copy()
            nrun = rng.poisson(n_frac * len(a) / 20.0)
            for _ in range(nrun):
                p = int(rng.integers(0, len(a)))
                a[p:p + int(rng.integers(1, 40))] = ord("N")
        seqs.append(a.tobytes())
    large, small = seqs[:n_contigs], seqs[n_contigs:]
    if n_samples > 0:
        gmean = np.exp(rng.normal(2.0, 1.0, size=(n_genomes, n_samples)))
        if absent_frac > 0.0:
            gmean[rng.random((n_genomes, n_samples)) < absent_frac] = 0.0
        depth = rng.poisson(gmean[genome_of]).astype(np.float32)
    else:
        depth = np.zeros((n_contigs, 0), dtype=np.float32)
    names = [f"contig_{i}" for i in range(n_contigs)]
    return Assembly(seqs=large, depth=depth, genome_of=genome_of,
                    small_seqs=small, names=names)


def write_fasta(asm: Assembly, path: str):
    with open(path, "wb") as f:
        for i, s in enumerate(asm.seqs):
            f.write(b">" + asm.names[i].encode() + b"\n")
            for p in range(0, len(s), 80):
                f.write(s[p:p + 80] + b"\n")
        for i, s in enumerate(asm.small_seqs):
            f.write(f">small_{i}\n".encode())
            for p in range(0, len(s), 80):
                f.write(s[p:p + 80] + b"\n")


def write_depth(asm: Assembly, path: str):
    """MetaBAT/JGI layout: contigName contigLen totalAvgDepth {mean var} x S."""
    S = asm.n_samples
    with open(path, "w") as f:
        hdr = ["contigName", "contigLen", "totalAvgDepth"]
        for s in range(S):
            hdr += [f"s{s}.bam", f"s{s}.bam-var"]
        f.write("\t".join(hdr) + "\n")
        for i, s in enumerate(asm.seqs):
            row = [asm.names[i], str(len(s)), f"{float(asm.depth[i].sum()):.6g}"]
            for k in range(S):
                v = float(asm.depth[i, k])
                row += [f"{v:.6g}", f"{v:.6g}"]
            f.write("\t".join(row) + "\n")


# ── synthetic BAM files (depth summariser) ─────────────────────────────────
_BAM_OPT_FIELDS = [("seed", "u64"), ("read_len", "i32"), ("level", "i32"), ("straddle", "i32"),
                   ("n_unmapped_tail", "i32"),
                   ("p_indel", "f64"), ("p_soft", "f64"), ("p_overhang", "f64"),
                   ("p_secondary", "f64"), ("p_dup", "f64"), ("p_qcfail", "f64"),
                   ("p_unmapped", "f64"), ("p_badmate", "f64"), ("p_nonm", "f64"),
                   ("p_lowq", "f64"), ("p_eqx", "f64"), ("p_mixed", "f64"), ("p_nm_off", "f64"),
                   ("err_mean", "f64")]

# the variety of reads the tests use; the benchmark keeps mostly clean reads
BAM_EDGE_CASES = dict(p_indel=0.15, p_soft=0.1, p_overhang=0.05, p_secondary=0.03, p_dup=0.03,
                      p_qcfail=0.02, p_unmapped=0.02, p_badmate=0.03, p_nonm=0.03, p_lowq=0.1,
                      p_eqx=0.15, p_mixed=0.1, p_nm_off=0.05, err_mean=0.02)
BAM_CLEAN = dict(p_indel=0.05, p_soft=0.05, p_overhang=0.0, p_secondary=0.01, p_dup=0.01,
                 p_qcfail=0.0, p_unmapped=0.005, p_badmate=0.0, p_nonm=0.0, p_lowq=0.05,
                 p_eqx=0.0, p_mixed=0.0, p_nm_off=0.0, err_mean=0.01)


def make_bam(lengths, depth, names=None, seq=None, seq_off=None, seed=1, read_len=150,
             level=6, straddle=False, n_unmapped_tail=50, **probs) -> bytes:
    """A coordinate-sorted BAM (BGZF bytes) of reads over contigs of the given
    lengths at the given mean depths (one value per contig).  `probs` override
    the read-variety probabilities of BAM_EDGE_CASES; `seq` / `seq_off` (ASCII
    bases and n+1 offsets) make the reads' bases those of the contigs."""
    import ctypes
    lengths = np.ascontiguousarray(lengths, dtype=np.uint32)
    n = len(lengths)
    depth = np.ascontiguousarray(depth, dtype=np.float32)
    assert depth.shape == (n,)
    if names is None:
        names = [f"contig_{i}" for i in range(n)]
    nb = b"".join(s.encode() + b"\0" for s in names) or b"\0"
    vals = dict(BAM_EDGE_CASES)
    vals.update(probs)
    vals.update(seed=seed, read_len=read_len, level=level, straddle=int(bool(straddle)),
                n_unmapped_tail=n_unmapped_tail)

    class Opts(ctypes.Structure):
        _fields_ = [(k, {"u64": ctypes.c_uint64, "i32": ctypes.c_int32, "f64": ctypes.c_double}[t])
                    for k, t in _BAM_OPT_FIELDS]

    o = Opts(**{k: vals[k] for k, _ in _BAM_OPT_FIELDS})
    lib = _chain_so()
    lib.synth_bam.restype = ctypes.c_int64
    out = ctypes.POINTER(ctypes.c_uint8)()
    P = ctypes.c_void_p
    if seq is not None:
        seq = (np.frombuffer(seq, dtype=np.uint8) if isinstance(seq, (bytes, bytearray))
               else np.ascontiguousarray(seq, dtype=np.uint8))
        seq_off = np.ascontiguousarray(seq_off, dtype=np.int64)
    size = lib.synth_bam(ctypes.byref(o), ctypes.c_int32(n), P(lengths.ctypes.data), nb,
                         P(depth.ctypes.data), P(seq.ctypes.data) if seq is not None else None,
                         P(seq_off.ctypes.data) if seq is not None else None, ctypes.byref(out))
    data = ctypes.string_at(out, size)
    lib.synth_bam_free(out)
    return data


def bam_records(bam: bytes):
    """(records, target lengths, names) of a BAM: the decompressed bytes after
    the header (each record: block_size, then the record), for the oracle."""
    import zlib
    mv = memoryview(bam)
    parts, o = [], 0
    while o < len(bam):                     # BGZF members, by their BC size field
        bsize = int.from_bytes(bam[o + 16:o + 18], "little") + 1
        parts.append(zlib.decompress(mv[o + 18:o + bsize - 8], -15))
        o += bsize
    raw = b"".join(parts)
    assert raw[:4] == b"BAM\1"
    l_text = int.from_bytes(raw[4:8], "little")
    o = 8 + l_text
    n_ref = int.from_bytes(raw[o:o + 4], "little")
    o += 4
    tl, nm = [], []
    for _ in range(n_ref):
        ln = int.from_bytes(raw[o:o + 4], "little")
        nm.append(raw[o + 4:o + 4 + ln].rstrip(b"\0").decode())
        tl.append(int.from_bytes(raw[o + 4 + ln:o + 8 + ln], "little"))
        o += 8 + ln
    return raw[o:], np.asarray(tl, dtype=np.uint32), nm
