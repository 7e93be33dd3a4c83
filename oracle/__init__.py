"""ctypes bindings of the oracle libraries (test infrastructure only).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this
package.  ``ref()`` is RabbitBin's own code compiled from the reference tree
(see build.py); ``restated()`` is the plain CPU restatement in rb_oracle.cpp.
"""
import ctypes as C
import os

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))


class RefParams(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int32), ("S", C.c_int32),
                ("win_bits", C.c_int32), ("max_edges", C.c_int32),
                ("mutual", C.c_int32), ("base_on", C.c_int32),
                ("nthreads", C.c_int32), ("seed", C.c_uint32),
                ("force_path", C.c_int32), ("coverage", C.c_double),
                ("min_edge", C.c_double), ("w_comp", C.c_double),
                ("min_cv", C.c_double), ("neg_thr", C.c_double),
                ("depth_sim", C.c_int32), ("depth_fuse", C.c_int32),
                ("wjac_norm", C.c_int32), ("no_abdfirst", C.c_int32),
                ("oph_k", C.c_int32), ("oph_bits", C.c_int32),
                ("graph_index", C.c_int32), ("min_common", C.c_int32), ("index_k", C.c_int32)]


class RefOut(C.Structure):
    _fields_ = [("b0", C.c_double), ("sim_cutoff", C.c_double),
                ("n_edges", C.c_int64),
                ("from_", C.POINTER(C.c_uint32)), ("to", C.POINTER(C.c_uint32)),
                ("scomp", C.POINTER(C.c_float)), ("score", C.POINTER(C.c_float))]


def default_params(n, m=500, S=0, **kw):
    p = RefParams(n=n, m=m, S=S, win_bits=16, max_edges=200, mutual=1,
                  base_on=1, nthreads=os.cpu_count() or 1, seed=1, force_path=0,
                  coverage=0.95, min_edge=0.70, w_comp=-1.0, min_cv=1.0,
                  neg_thr=-0.3, depth_sim=2, depth_fuse=1, wjac_norm=1, no_abdfirst=0,
                  oph_k=0, oph_bits=2, graph_index=0, min_common=0, index_k=8)
    if "abdfirst" in kw:
        kw["no_abdfirst"] = 0 if kw.pop("abdfirst") else 1
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class _Lib:
    """Common wrappers over the harness / restatement entry points."""

    def __init__(self, path, prefix):
        self.lib = C.CDLL(path)
        self.path = path
        L, p = self.lib, prefix
        self._bw = getattr(L, p + "build_winners")
        self._bw.restype = None
        self._bw.argtypes = [C.c_char_p, C.POINTER(C.c_int64), C.c_int64, C.c_int,
                             C.c_uint32, C.c_uint64, C.c_int, C.c_double,
                             C.POINTER(C.c_uint32), C.c_int]
        self._rg = getattr(L, p + "run_graph")
        self._rg.restype = C.c_int
        self._rg.argtypes = [C.POINTER(RefParams), C.POINTER(C.c_uint32),
                             C.POINTER(C.c_float), C.POINTER(C.c_float),
                             C.POINTER(RefOut)]
        self._free = getattr(L, p + "free")
        self._free.argtypes = [C.c_void_p]
        self._pe = getattr(L, p + "pmh_elements")
        self._pe.restype = None
        self._pe.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_int64,
                             C.c_uint32, C.c_uint64, C.POINTER(C.c_double),
                             C.POINTER(C.c_uint64)]
        self._ud = getattr(L, p + "unit_dot_f")
        self._ud.restype = C.c_float
        self._ud.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_uint32]
        self._ov = getattr(L, p + "oph_values")
        self._ov.restype = None
        self._ov.argtypes = [C.c_char_p, C.POINTER(C.c_int64), C.c_int64, C.c_uint32, C.c_int,
                             C.c_uint32, C.POINTER(C.c_uint8)]
        self._rgo = getattr(L, p + "run_graph_oph", None)
        if self._rgo is not None:
            self._rgo.restype = C.c_int
            self._rgo.argtypes = [C.POINTER(RefParams), C.c_char_p, C.POINTER(C.c_int64),
                                  C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(RefOut)]

    def label_propagation(self, n, src, dst, score, seed=1, node_order=None, nthreads=0):
        """cluster_by_propagation of the reference on an edge list (harness
        only): membership uint32[n].  The score rule follows RABBIT_LPA_SCORE
        as it was when the library loaded; RABBIT_PAR_LPA is read per call."""
        f = getattr(self.lib, "ref_label_propagation")
        f.restype = C.c_int
        f.argtypes = [C.c_int64, C.c_int64, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                      C.POINTER(C.c_float), C.c_ulonglong, C.POINTER(C.c_uint32),
                      C.POINTER(C.c_uint32), C.c_int]
        a = np.ascontiguousarray(src, np.uint32)
        b = np.ascontiguousarray(dst, np.uint32)
        w = np.ascontiguousarray(score, np.float32)
        order = None if node_order is None else np.ascontiguousarray(node_order, np.uint32)
        out = np.zeros(int(n), np.uint32)
        rc = f(int(n), len(a), _ptr(a, C.c_uint32), _ptr(b, C.c_uint32), _ptr(w, C.c_float),
               int(seed), None if order is None else _ptr(order, C.c_uint32),
               _ptr(out, C.c_uint32), int(nthreads))
        if rc != 0:
            raise ValueError("edgeScore must be non-negative")
        return out

    def lpa_node_order(self, n, seed=1):
        """The seeded node order of the reference (src/rabbitbin.cpp:5643-5645)."""
        f = getattr(self.lib, "ref_lpa_node_order")
        f.restype = None
        f.argtypes = [C.c_int64, C.c_ulonglong, C.POINTER(C.c_uint32)]
        out = np.zeros(int(n), np.uint32)
        f(int(n), int(seed), _ptr(out, C.c_uint32))
        return out

    def oph_values(self, seqcat, offsets, m=500, K=8, bits=2):
        """One-permutation MinHash bucket values [n, m] (uint8)."""
        n = len(offsets) - 1
        out = np.zeros((n, m), dtype=np.uint8)
        offs = np.ascontiguousarray(offsets, dtype=np.int64)
        self._ov(seqcat, _ptr(offs, C.c_int64), n, m, K, bits, _ptr(out, C.c_uint8))
        return out

    def build_winners(self, seqcat, offsets, k=4, m=500, seed=42, gc_norm=1,
                      gc_cap=20.0, nthreads=None):
        n = len(offsets) - 1
        out = np.zeros((n, m), dtype=np.uint32)
        offs = np.ascontiguousarray(offsets, dtype=np.int64)
        self._bw(seqcat, _ptr(offs, C.c_int64), n, k, m, seed, gc_norm, gc_cap,
                 _ptr(out, C.c_uint32), nthreads or os.cpu_count() or 1)
        return out

    def run_graph(self, params, winners32, depth):
        n, S = params.n, params.S
        w = np.ascontiguousarray(winners32, dtype=np.uint32)
        d = np.ascontiguousarray(depth, dtype=np.float32).reshape(n, max(S, 0))
        unit = np.zeros((n, max(S, 1)), dtype=np.float32)
        out = RefOut()
        rc = self._rg(C.byref(params), _ptr(w, C.c_uint32), _ptr(d, C.c_float),
                      _ptr(unit, C.c_float), C.byref(out))
        if rc != 0:
            raise RuntimeError(f"oracle run_graph failed: {rc}")
        return self._result(out, unit, S)

    def run_graph_index(self, params, seqcat, offsets, winners32, depth):
        """The small path with RABBIT_GRAPH_INDEX=1 (harness only): candidates
        from the inverted index of one-permutation sketch keys."""
        f = self.lib.ref_run_graph_index
        f.restype = C.c_int
        f.argtypes = [C.POINTER(RefParams), C.c_char_p, C.POINTER(C.c_int64),
                      C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.POINTER(C.c_float),
                      C.POINTER(RefOut)]
        n, S = params.n, params.S
        offs = np.ascontiguousarray(offsets, dtype=np.int64)
        w = np.ascontiguousarray(winners32, dtype=np.uint32)
        d = np.ascontiguousarray(depth, dtype=np.float32).reshape(n, max(S, 0))
        unit = np.zeros((n, max(S, 1)), dtype=np.float32)
        out = RefOut()
        rc = f(C.byref(params), seqcat, _ptr(offs, C.c_int64), _ptr(w, C.c_uint32),
               _ptr(d, C.c_float), _ptr(unit, C.c_float), C.byref(out))
        if rc != 0:
            raise RuntimeError(f"oracle run_graph_index failed: {rc}")
        return self._result(out, unit, S)

    def run_graph_oph(self, params, seqcat, offsets, depth):
        """The graph with RABBIT_PMH=0 (params.oph_k, params.oph_bits set)."""
        n, S = params.n, params.S
        offs = np.ascontiguousarray(offsets, dtype=np.int64)
        d = np.ascontiguousarray(depth, dtype=np.float32).reshape(n, max(S, 0))
        unit = np.zeros((n, max(S, 1)), dtype=np.float32)
        out = RefOut()
        rc = self._rgo(C.byref(params), seqcat, _ptr(offs, C.c_int64), _ptr(d, C.c_float),
                       _ptr(unit, C.c_float), C.byref(out))
        if rc != 0:
            raise RuntimeError(f"oracle run_graph_oph failed: {rc}")
        return self._result(out, unit, S)

    def _result(self, out, unit, S):
        ne = out.n_edges
        res = dict(b0=out.b0, sim_cutoff=out.sim_cutoff,
                   src=np.ctypeslib.as_array(out.from_, (ne,)).copy() if ne else np.zeros(0, np.uint32),
                   dst=np.ctypeslib.as_array(out.to, (ne,)).copy() if ne else np.zeros(0, np.uint32),
                   scomp=np.ctypeslib.as_array(out.scomp, (ne,)).copy() if ne else np.zeros(0, np.float32),
                   score=np.ctypeslib.as_array(out.score, (ne,)).copy() if ne else np.zeros(0, np.float32),
                   unit=unit[:, :S] if S > 1 else None)
        for ptr in (out.from_, out.to, out.scomp, out.score):
            self._free(C.cast(ptr, C.c_void_p))
        return res

    def pmh_elements(self, keys, weights, m=500, seed=42):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        regs = np.zeros(m, dtype=np.float64)
        win = np.zeros(m, dtype=np.uint64)
        self._pe(_ptr(keys, C.c_uint64), _ptr(w, C.c_double), len(keys), m, seed,
                 _ptr(regs, C.c_double), _ptr(win, C.c_uint64))
        return regs, win

    def pmh_metrics(self, ka, wa, kb, wb, m=500, seed=42, kmer=4):
        """(jaccard_weighted, jaccard, distance, ani) of two ProbMinHash4
        sketches built from element sets, by the reference's own methods
        (harness only)."""
        f = self.lib.ref_pmh_metrics
        f.restype = None
        f.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_int64,
                      C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_int64, C.c_uint32,
                      C.c_uint64, C.c_int, C.POINTER(C.c_double)]
        ka = np.ascontiguousarray(ka, np.uint64)
        kb = np.ascontiguousarray(kb, np.uint64)
        wa = np.ascontiguousarray(wa, np.float64)
        wb = np.ascontiguousarray(wb, np.float64)
        out = np.zeros(4, np.float64)
        f(_ptr(ka, C.c_uint64), _ptr(wa, C.c_double), len(ka), _ptr(kb, C.c_uint64),
          _ptr(wb, C.c_double), len(kb), m, seed, kmer, _ptr(out, C.c_double))
        return tuple(out)

    def unit_dot_f(self, a, b):
        a = np.ascontiguousarray(a, dtype=np.float32)
        b = np.ascontiguousarray(b, dtype=np.float32)
        return float(self._ud(_ptr(a, C.c_float), _ptr(b, C.c_float), len(a)))


_cache = {}


def ref():
    """RabbitBin's own hot-path code (None when not built and not buildable)."""
    if "ref" not in _cache:
        path = _build.build_ref()
        _cache["ref"] = _Lib(path, "ref_") if path and os.path.exists(path) else None
    return _cache["ref"]


def restated():
    """The CPU restatement of the hot path (always available)."""
    if "orc" not in _cache:
        _cache["orc"] = _Lib(_build.build_oracle(), "orc_")
    return _cache["orc"]


def sorted_edges(res):
    """Edge set sorted by (src, dst): the reference emits rows in thread order."""
    order = np.lexsort((res["dst"], res["src"]))
    return (res["src"][order], res["dst"][order], res["scomp"][order],
            res["score"][order])


class _RefFasta(C.Structure):
    _fields_ = [("num_seqs", C.c_int64), ("n_large", C.c_int64), ("n_small", C.c_int64),
                ("names", C.c_void_p), ("name_off", C.POINTER(C.c_int64)),
                ("seqcat", C.c_void_p), ("seq_off", C.POINTER(C.c_int64))]


class _OrcFasta(C.Structure):
    _fields_ = [("num_seqs", C.c_int64), ("n_large", C.c_int64), ("n_small", C.c_int64),
                ("name_start", C.POINTER(C.c_int64)), ("name_len", C.POINTER(C.c_int32)),
                ("seq", C.c_void_p), ("seq_off", C.POINTER(C.c_int64))]


def _split(base, off, count):
    return [C.string_at(base + off[i], off[i + 1] - off[i]) for i in range(count)]


def parse_fasta_ref(path, min_contig=2500, min_small=1000, nthreads=4):
    """RabbitBin's own parse_fasta_mmap_parallel on a file (None if the
    harness is not built): {num_seqs, large: [(name, seq)], small: [...]}."""
    lib = ref()
    if lib is None:
        return None
    f = lib.lib.ref_parse_fasta
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.c_int, C.c_int64, C.c_int64, C.POINTER(_RefFasta)]
    out = _RefFasta()
    if f(path.encode(), nthreads, min_contig, min_small, C.byref(out)) != 0:
        raise RuntimeError("reference parser failed")
    n = out.n_large + out.n_small
    names = _split(out.names, out.name_off, n)
    seqs = _split(out.seqcat, out.seq_off, n)
    for p in (out.names, out.seqcat, C.cast(out.name_off, C.c_void_p).value,
              C.cast(out.seq_off, C.c_void_p).value):
        lib._free(p)
    pairs = list(zip(names, seqs))
    return {"num_seqs": out.num_seqs, "large": pairs[:out.n_large], "small": pairs[out.n_large:]}


def parse_fasta_restated(data, min_contig=2500, min_small=1000):
    """The restated parser on an in-memory file; same result shape."""
    lib = restated()
    f = lib.lib.orc_parse_fasta
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.POINTER(_OrcFasta)]
    out = _OrcFasta()
    f(data, len(data), min_contig, min_small, C.byref(out))
    n = out.n_large + out.n_small
    names = [data[out.name_start[i]:out.name_start[i] + out.name_len[i]] for i in range(n)]
    seqs = _split(out.seq, out.seq_off, n)
    for p in (out.seq, C.cast(out.name_start, C.c_void_p).value,
              C.cast(out.name_len, C.c_void_p).value, C.cast(out.seq_off, C.c_void_p).value):
        lib._free(p)
    pairs = list(zip(names, seqs))
    return {"num_seqs": out.num_seqs, "large": pairs[:out.n_large], "small": pairs[out.n_large:]}


def fp64_edge_weights(depth, src, dst, scomp, w_comp=-1.0, min_edge=0.70, neg_thr=-0.3,
                      wjac_norm=True, chunk=1 << 20, margins=False):
    """Edge weights in FP64 from the raw coverage (the tolerance oracle).

    The edge-weight loop of src/rabbitbin.cpp:5482-5509 with depth_edge_term
    (:930-970) in its default mode (RABBIT_DEPTH_SIM=2, fuse = min): average
    ranks of each contig's S coverage values (src/ranker.h:55-66), centred and
    L2-normalised (:4972-4988), their dot product as the rank correlation, the
    weighted Jaccard of the column-normalised raw depths (:685-698, column norm
    1/mean :4792-4809), dterm = min(max(rho, 0), clip(wJ)), w = a*sComp +
    (1-a)*dterm with a = 1 for S <= 2 else 0 (auto_w_comp :470-473), cut to 0
    when rho < neg_thr or w < min_edge.  Everything is evaluated in double,
    nothing stored as float, so the device weights' distance to these values is
    their FP32 error.  Returns float64[E] (sComp itself when S <= 1); with
    margins=True also each edge's FP64 distance to the nearer cut threshold
    (|w - min_edge|, |rho - neg_thr|)."""
    from scipy.stats import rankdata
    d = np.ascontiguousarray(depth, dtype=np.float32).astype(np.float64)
    n = d.shape[0]
    S = d.shape[1] if d.ndim == 2 else 0
    scomp = np.asarray(scomp, dtype=np.float64)
    if S <= 1:
        return (scomp.copy(), np.full(len(scomp), np.inf)) if margins else scomp.copy()
    r = rankdata(d, axis=1, method="average")
    r -= r.mean(axis=1, keepdims=True)
    ss = np.sqrt((r * r).sum(axis=1, keepdims=True))
    u = np.divide(r, ss, out=np.zeros_like(r), where=ss > 0)
    if wjac_norm:
        mean = d.sum(axis=0) / max(n, 1)
        cn = np.where(mean > 1e-12, 1.0 / np.where(mean > 1e-12, mean, 1.0), 0.0)
    else:
        cn = np.ones(S)
    a = (1.0 if S <= 2 else 0.0) if w_comp < 0 else float(w_comp)
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    out = np.zeros(len(src), dtype=np.float64)
    marg = np.full(len(src), np.inf)
    for b in range(0, len(src), chunk):
        i, j = src[b:b + chunk], dst[b:b + chunk]
        rho = np.einsum("ij,ij->i", u[i], u[j])
        x, y = d[i] * cn, d[j] * cn
        mx = np.maximum(x, y).sum(axis=1)
        wj = np.divide(np.minimum(x, y).sum(axis=1), mx, out=np.zeros_like(mx), where=mx > 0)
        wj = np.clip(wj, 0.0, 1.0)
        dterm = np.minimum(np.maximum(rho, 0.0), wj)
        w = a * scomp[b:b + chunk] + (1.0 - a) * dterm
        cut = (w < min_edge) | ((rho < neg_thr) if neg_thr > -0.99 else False)
        out[b:b + chunk] = np.where(cut, 0.0, w)
        mg = np.abs(w - min_edge)
        if neg_thr > -0.99:
            mg = np.minimum(mg, np.abs(rho - neg_thr))
        marg[b:b + chunk] = mg
    return (out, marg) if margins else out


def fp64_report(depth, g, **kw):
    """{max_abs_err_fp64, edges, cut_disagreements, max_margin_disagreeing} of
    a graph's edge weights against fp64_edge_weights.  The error is taken over
    the edges on whose cut the two agree.  cut_disagreements counts the edges
    that one side keeps and the other cuts: values that sit on a threshold in
    exact arithmetic (with S = 5 the rank correlation is a multiple of 1/20, so
    0.70 is reached exactly), where the FP32 rounding decides, as it does in
    the reference; max_margin_disagreeing is the largest FP64 distance of such
    an edge to its threshold (at most the FP32 error when the cut is a tie)."""
    fp, marg = fp64_edge_weights(depth, g["src"], g["dst"], g["scomp"], margins=True, **kw)
    got = np.asarray(g["score"], dtype=np.float64)
    agree = (fp > 0) == (got > 0)
    err = np.abs(fp[agree] - got[agree])
    dis = marg[~agree]
    return {"max_abs_err_fp64": float(err.max()) if err.size else 0.0,
            "edges": int(len(got)), "cut_disagreements": int((~agree).sum()),
            "max_margin_disagreeing": float(dis.max()) if dis.size else 0.0}


def ref_cache_write(path, state):
    """RabbitBin's own rb_write_cache of a state dict (harness only; the dict
    layout of rabbitbin_b200.api.cache_struct)."""
    from rabbitbin_b200 import api
    lib = ref()

    class RefCacheState(C.Structure):
        _fields_ = api._CACHE_FIELDS
    st, keep = api.cache_struct(RefCacheState, state)
    f = lib.lib.ref_cache_write
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.POINTER(RefCacheState)]
    if f(str(path).encode(), C.byref(st)) != 0:
        raise RuntimeError("reference rb_write_cache failed")


def ref_cache_read(path):
    """RabbitBin's own rb_load_cache of a file, as a state dict (harness
    only), or None when the reference rejects the file."""
    from rabbitbin_b200 import api
    lib = ref()

    class RefCacheState(C.Structure):
        _fields_ = api._CACHE_FIELDS
    f = lib.lib.ref_cache_read
    f.restype = C.c_int
    f.argtypes = [C.c_char_p, C.POINTER(RefCacheState)] + [C.c_void_p] * 17
    st = RefCacheState()
    if f(str(path).encode(), C.byref(st), *([None] * 17)) != 0:
        return None
    nl, ns = st.n_large_names, st.n_small_names
    bufs = {}
    # name bytes: the file size bounds them
    size = os.path.getsize(path)
    lnames, snames = np.zeros(size + 1, np.uint8), np.zeros(size + 1, np.uint8)
    lnoff, snoff = np.zeros(nl + 1, np.int64), np.zeros(ns + 1, np.int64)
    arrays = []
    for name, dt, cnt in api.CACHE_ARRAYS:
        n = getattr(st, cnt[0]) * getattr(st, cnt[1]) if isinstance(cnt, tuple) else getattr(st, cnt)
        bufs[name] = np.zeros(max(int(n), 1), dt)
        arrays.append(bufs[name].ctypes.data)
    args = [lnames.ctypes.data, lnoff.ctypes.data, snames.ctypes.data, snoff.ctypes.data] + arrays
    if f(str(path).encode(), C.byref(st), *args) != 0:
        return None
    out = {k: getattr(st, k) for k in api.CACHE_SCALARS}
    out["large_names"] = [lnames[lnoff[i]:lnoff[i + 1]].tobytes() for i in range(nl)]
    out["small_names"] = [snames[snoff[i]:snoff[i + 1]].tobytes() for i in range(ns)]
    for name, dt, cnt in api.CACHE_ARRAYS:
        if isinstance(cnt, tuple):
            r, c = getattr(st, cnt[0]), getattr(st, cnt[1])
            out[name] = bufs[name][:r * c].reshape(r, c)
        else:
            out[name] = bufs[name][:getattr(st, cnt)]
    return out


# ── BAM -> depth: the reference's per-read code (librbref_depth.so) ─────────
def ref_depth():
    """depth_accumulate_sample and the code under it, compiled from the
    reference tree (ref_depth_shim.cpp); None when neither built nor buildable."""
    if "depth" not in _cache:
        _build.build_ref()
        path = os.path.join(_HERE, "_ref", "librbref_depth.so")
        lib = None
        if os.path.exists(path):
            lib = C.CDLL(path)
            f = lib.ref_depth_accumulate
            f.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_uint32), C.c_int32, C.c_float,
                          C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64),
                          C.POINTER(C.c_int32)]
            f.restype = C.c_int
        _cache["depth"] = lib
    return _cache["depth"]


def depth_accumulate_ref(records, target_len, pctid=0.97, max_edge=75, include_edge=False,
                         min_mapq=0, threads=0):
    """(sums uint64[n_targets], avg_read) of depth_accumulate_sample
    (src/rabbit_depth.cpp:1615-1685) over decompressed records."""
    lib = ref_depth()
    if lib is None:
        return None
    rec = np.frombuffer(bytes(records), np.uint8) if len(records) else np.zeros(1, np.uint8)
    tl = np.ascontiguousarray(target_len, np.uint32)
    out = np.zeros(max(len(tl), 1), np.uint64)
    avg = C.c_int32(0)
    rc = lib.ref_depth_accumulate(rec.ctypes.data, len(records), _ptr(tl, C.c_uint32), len(tl),
                                  C.c_float(pctid), int(max_edge), int(bool(include_edge)),
                                  int(min_mapq), int(threads), _ptr(out, C.c_uint64),
                                  C.byref(avg))
    if rc != 0:
        raise ValueError("malformed records")
    return out[:len(tl)], int(avg.value)


def depth_means(sums, target_len, edge):
    """Means of src/rabbit_depth.cpp:1515-1534: (float)((double)sum / adj) with
    adj = len - 2 edge for len > 2 edge + 1 (else len), 0 for adj <= 2, values
    above 1e6 set to 0."""
    cl = np.asarray(target_len, np.uint32).astype(np.int32).astype(np.int64)
    adj = np.where(cl > 2 * edge + 1, cl - 2 * edge, cl)
    with np.errstate(divide="ignore", invalid="ignore"):
        m = (np.asarray(sums, np.uint64).astype(np.float64) / np.where(adj > 2, adj, 1)).astype(np.float32)
    m = np.where(adj > 2, m, np.float32(0))
    m[m > np.float32(1000000.0)] = 0
    return m.astype(np.float32)


def depth_tsv_ref(sums, avg, target_len, names, bam_names, variance=False, include_edge=False,
                  max_edge=75, min_contig_len=1, min_contig_depth=0.0):
    """printDepthTable's bytes (src/rabbit_depth.cpp:125-313) for per-BAM sums
    [n_bams, n_targets] and read lengths, as compute_depth_tsv_inmem calls it."""
    lib = ref_depth()
    if lib is None:
        return None
    f = lib.ref_depth_tsv
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_char_p, C.c_int32,
                  C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                  C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
    f.restype = C.c_int
    lib.ref_free.argtypes = [C.c_void_p]
    s = np.ascontiguousarray(sums, np.uint64)
    a = np.ascontiguousarray(avg, np.int32)
    tl = np.ascontiguousarray(target_len, np.uint32)
    nb = b"".join(x.encode() + b"\0" for x in names) or b"\0"
    bb = b"".join(x.encode() + b"\0" for x in bam_names)
    out, ln = C.c_void_p(), C.c_int64()
    f(s.ctypes.data, a.ctypes.data, len(a), tl.ctypes.data, nb, len(tl), bb, int(variance),
      int(include_edge), int(max_edge), int(min_contig_len), C.c_float(min_contig_depth),
      C.byref(out), C.byref(ln))
    r = C.string_at(out, ln.value)
    lib.ref_free(out)
    return r
