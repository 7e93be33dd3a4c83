"""Python binding of the C ABI in include/rabbitbin_b200.h (ctypes).

The product is the CUDA library ``librabbitbin_b200.so`` built in-tree by
``rabbitbin_b200.build``; this module only marshals host arrays.  There is no
CPU fallback: without a CUDA device every compute call raises ``RbgError``.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librabbitbin_b200.so")

RBG_OK = 0
_STATUS = {-1: "bad argument", -2: "out of memory", -3: "CUDA error",
           -4: "unsupported option", -5: "device wait timed out"}


class RbgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_STATUS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    """rbg_params: `rabbitbin bin` options and hot-path RABBIT_* settings."""
    _fields_ = [("k", C.c_int32), ("m", C.c_int32), ("pmh_seed", C.c_uint64),
                ("gc_norm", C.c_int32), ("win_bits", C.c_int32),
                ("gc_norm_cap", C.c_double), ("max_edges", C.c_int32),
                ("mutual", C.c_int32), ("base_on", C.c_int32), ("seed", C.c_uint32),
                ("force_path", C.c_int32), ("abdfirst", C.c_int32),
                ("coverage", C.c_double), ("min_edge", C.c_double),
                ("w_comp", C.c_double), ("min_cv", C.c_double), ("neg_thr", C.c_double),
                ("depth_sim", C.c_int32), ("depth_fuse", C.c_int32),
                ("wjac_norm", C.c_int32), ("fp_contract", C.c_int32),
                ("wjac_cut", C.c_double), ("wjac_gate", C.c_int32), ("oph_k", C.c_int32),
                ("oph_bits", C.c_int32), ("graph_index", C.c_int32), ("index_k", C.c_int32),
                ("min_common", C.c_int32), ("reserved", C.c_int32)]


class Graph(C.Structure):
    _fields_ = [("n_edges", C.c_int64), ("from_", C.POINTER(C.c_uint32)),
                ("to", C.POINTER(C.c_uint32)), ("scomp", C.POINTER(C.c_float)),
                ("score", C.POINTER(C.c_float)), ("b0", C.c_double),
                ("sim_cutoff", C.c_double), ("path", C.c_int32), ("reserved", C.c_int32)]


class Timing(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("pack_ms", "count_ms", "sketch_ms", "unit_ms",
                                        "b0_ms", "allpairs_ms", "finalize_ms", "emit_ms",
                                        "weight_ms", "total_ms")] + \
               [("pairs_prefiltered", C.c_int64), ("pairs_compared", C.c_int64),
                ("kernel_launches", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


class Assembly(C.Structure):
    """rbg_assembly: one assembly of a batch (host arrays)."""
    _fields_ = [("seqcat", C.c_char_p), ("offsets", C.POINTER(C.c_int64)), ("n", C.c_int64),
                ("depth", C.POINTER(C.c_float)), ("S", C.c_int32), ("reserved", C.c_int32),
                ("params", C.POINTER(Params))]


class BatchStats(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("stage_ms", "graph_ms", "calib_ms", "emit_ms",
                                        "total_ms")] + \
               [("n_assemblies", C.c_int32), ("kernel_launches", C.c_int32),
                ("graph_launches", C.c_int32), ("tuned_keys", C.c_int32),
                ("rows", C.c_int64), ("pairs", C.c_int64), ("items", C.c_int64),
                ("edges", C.c_int64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


class Fasta(C.Structure):
    _fields_ = [("num_seqs", C.c_int64), ("n_large", C.c_int64), ("n_small", C.c_int64),
                ("large_seq", C.c_void_p), ("large_off", C.POINTER(C.c_int64)),
                ("large_name_start", C.POINTER(C.c_int64)), ("large_name_len", C.POINTER(C.c_int32)),
                ("small_seq", C.c_void_p), ("small_off", C.POINTER(C.c_int64)),
                ("small_name_start", C.POINTER(C.c_int64)), ("small_name_len", C.POINTER(C.c_int32))]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("workers", C.c_int32), ("hbm_budget", C.c_int64),
                ("max_batch", C.c_int32), ("plain", C.c_int32), ("max_batch_pairs", C.c_int64),
                ("small_pairs", C.c_int64)]


class RequestStats(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("service_ms", C.c_double), ("latency_ms", C.c_double),
                ("batch_size", C.c_int32), ("worker", C.c_int32), ("est_bytes", C.c_int64),
                ("submit_s", C.c_double), ("done_s", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_CACHE_FIELDS = [
    ("n_large", C.c_int64), ("n_small", C.c_int64), ("samples", C.c_int64),
    ("seed", C.c_uint64), ("total_size", C.c_uint64), ("total_size_small", C.c_uint64),
    ("sim_cutoff", C.c_double), ("b0", C.c_double),
    ("min_contig", C.c_uint64), ("min_small_contig", C.c_uint64),
    ("has_depth", C.c_int32), ("has_snv", C.c_int32),
    ("large_names", C.c_void_p), ("large_name_off", C.c_void_p), ("n_large_names", C.c_int64),
    ("small_names", C.c_void_p), ("small_name_off", C.c_void_p), ("n_small_names", C.c_int64),
    ("large_len", C.c_void_p), ("n_large_len", C.c_int64),
    ("small_len", C.c_void_p), ("n_small_len", C.c_int64),
    ("depth_ranked", C.c_void_p), ("depth_rows", C.c_int64), ("depth_cols", C.c_int64),
    ("small_depth", C.c_void_p), ("small_depth_rows", C.c_int64), ("small_depth_cols", C.c_int64),
    ("large_means", C.c_void_p), ("n_large_means", C.c_int64),
    ("depth_raw", C.c_void_p), ("n_depth_raw", C.c_int64),
    ("colnorm", C.c_void_p), ("n_colnorm", C.c_int64),
    ("from_", C.c_void_p), ("to", C.c_void_p), ("scomp", C.c_void_p), ("n_edges", C.c_int64),
    ("snv_pi", C.c_void_p), ("snv_nsnv", C.c_void_p), ("snv_cov", C.c_void_p),
    ("n_snv", C.c_int64)]


class CacheState(C.Structure):
    """rbg_cache: the state stored in an RBCACHE1 file."""
    _fields_ = _CACHE_FIELDS + [("version", C.c_int32), ("reserved", C.c_int32)]


# (field, numpy dtype, count field or (rows, cols)) of every array of the state
CACHE_ARRAYS = [("large_len", np.uint64, "n_large_len"), ("small_len", np.uint64, "n_small_len"),
                ("depth_ranked", np.float32, ("depth_rows", "depth_cols")),
                ("small_depth", np.float32, ("small_depth_rows", "small_depth_cols")),
                ("large_means", np.float32, "n_large_means"),
                ("depth_raw", np.float32, "n_depth_raw"), ("colnorm", np.float64, "n_colnorm"),
                ("from_", np.uint32, "n_edges"), ("to", np.uint32, "n_edges"),
                ("scomp", np.float32, "n_edges"), ("snv_pi", np.float32, "n_snv"),
                ("snv_nsnv", np.uint32, "n_snv"), ("snv_cov", np.uint32, "n_snv")]
CACHE_SCALARS = ["n_large", "n_small", "samples", "seed", "total_size", "total_size_small",
                 "sim_cutoff", "b0", "min_contig", "min_small_contig", "has_depth", "has_snv"]


def cache_struct(cls, state):
    """A ctypes state of class `cls` pointing into numpy copies of `state`
    (dict: the scalars, 'large_names' / 'small_names' lists of bytes, the
    arrays); returns (struct, keep-alive list)."""
    st, keep = cls(), []
    for k in CACHE_SCALARS:
        setattr(st, k, state.get(k, 0))
    for key in ("large_names", "small_names"):
        names = state.get(key) or []
        off = np.zeros(len(names) + 1, np.int64)
        off[1:] = np.cumsum([len(x) for x in names])
        buf = np.frombuffer(b"".join(names) + b"\0", np.uint8).copy()
        keep += [buf, off]
        setattr(st, key, buf.ctypes.data if names else None)
        setattr(st, key.replace("names", "name_off"), off.ctypes.data if names else None)
        setattr(st, "n_" + key, len(names))
    for name, dt, cnt in CACHE_ARRAYS:
        a = state.get(name)
        if a is None:
            a = np.zeros(0, dt)
        a = np.ascontiguousarray(a, dt)
        keep.append(a)
        setattr(st, name, a.ctypes.data if a.size else None)
        if isinstance(cnt, tuple):
            r, c = (a.shape if a.ndim == 2 else (0, 0))
            setattr(st, cnt[0], r)
            setattr(st, cnt[1], c)
        else:
            setattr(st, cnt, a.size)
    return st, keep


def cache_dict(st):
    """The state of a filled ctypes struct as a dict of copies."""
    out = {k: getattr(st, k) for k in CACHE_SCALARS}
    for key in ("large_names", "small_names"):
        n = getattr(st, "n_" + key)
        base, off = getattr(st, key), getattr(st, key.replace("names", "name_off"))
        if n and base:
            o = np.ctypeslib.as_array(C.cast(off, C.POINTER(C.c_int64)), (n + 1,))
            out[key] = [C.string_at(base + int(o[i]), int(o[i + 1] - o[i])) for i in range(n)]
        else:
            out[key] = []
    for name, dt, cnt in CACHE_ARRAYS:
        p = getattr(st, name)
        shape = (getattr(st, cnt[0]), getattr(st, cnt[1])) if isinstance(cnt, tuple) \
            else (getattr(st, cnt),)
        size = int(np.prod(shape))
        if p and size:
            ct = np.ctypeslib.as_ctypes_type(dt)
            out[name] = np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape).copy()
        else:
            out[name] = np.zeros(shape if isinstance(cnt, tuple) else (0,), dt)
    return out


def write_cache(path, state):
    """rbg_write_cache of a state dict (see cache_struct)."""
    st, keep = cache_struct(CacheState, state)
    rc = lib().rbg_write_cache(str(path).encode(), C.byref(st))
    if rc != RBG_OK:
        raise RbgError(rc, f"cannot write the cache {path}")


def read_cache(path):
    """rbg_read_cache as a state dict (plus 'version')."""
    st = CacheState()
    L = lib()
    rc = L.rbg_read_cache(str(path).encode(), C.byref(st))
    if rc != RBG_OK:
        raise RbgError(rc, f"cannot read the cache {path}")
    try:
        d = cache_dict(st)
        d["version"] = st.version
        return d
    finally:
        L.rbg_free_cache(C.byref(st))


_lib = None


# The collective of a sharded call: (send, recv, bytes_per_rank, user) -> 0 on success.
ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p)


class LpaParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("node_order", C.c_void_p), ("score_rule", C.c_int32),
                ("synchronous", C.c_int32), ("max_rounds", C.c_int32), ("reserved", C.c_int32)]


class LpaStats(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("reserved", C.c_int32), ("changes", C.c_int64),
                ("frozen", C.c_int64), ("arcs", C.c_int64), ("incidence_ms", C.c_float),
                ("sweep_ms", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# RABBIT_LPA_SCORE names (src/impl/rb_cluster.cpp:41-50) -> RBG_LPA_*
LPA_RULES = {"fisher": 0, "tail": 1, "logsum": 2, "sum": 3, "mean": 4, "max": 5}


class DepthParams(C.Structure):
    _fields_ = [("percent_identity", C.c_float), ("min_contig_length", C.c_int32),
                ("max_edge_bases", C.c_int32), ("include_edge_bases", C.c_int32),
                ("min_map_qual", C.c_int32), ("dual_map_qual", C.c_int32),
                ("threads", C.c_int32), ("chunk_mb", C.c_int32), ("device_inflate", C.c_int32),
                ("device_chunk_mb", C.c_int32)]


class DepthMatrix(C.Structure):
    _fields_ = [("n_rows", C.c_int64), ("n_cols", C.c_int32), ("n_targets", C.c_int32),
                ("tid", C.POINTER(C.c_int32)), ("lens", C.POINTER(C.c_int32)),
                ("means", C.POINTER(C.c_float)), ("names", C.c_void_p),
                ("name_off", C.POINTER(C.c_int64)), ("avg_read", C.POINTER(C.c_int32)),
                ("sums", C.POINTER(C.c_uint64)), ("records", C.c_int64),
                ("compressed_bytes", C.c_int64), ("decompressed_bytes", C.c_int64),
                ("inflate_ms", C.c_float), ("total_ms", C.c_float), ("kernel_ms", C.c_float),
                ("device_bams", C.c_int32)]


class Shard(C.Structure):
    _fields_ = [("rank", C.c_int32), ("world", C.c_int32), ("device_buffers", C.c_int32),
                ("reserved", C.c_int32), ("allgather", ALLGATHER_FN), ("user", C.c_void_p)]


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RbgError(-4, f"{LIB_PATH} is missing; run python -m rabbitbin_b200.build")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp, i64p = C.c_void_p, P(C.c_int64)
    sig = {
        "rbg_default_params": ([P(Params)], C.c_int),
        "rbg_create": ([C.c_int, P(vp)], C.c_int),
        "rbg_destroy": ([vp], C.c_int),
        "rbg_last_error": ([vp], C.c_char_p),
        "rbg_stream": ([vp], vp),
        "rbg_build_pmh_winners": ([vp, P(Params), C.c_char_p, i64p, C.c_int64,
                                   P(C.c_uint32)], C.c_int),
        "rbg_build_oph_signature": ([vp, P(Params), C.c_char_p, i64p, C.c_int64,
                                     P(C.c_uint8)], C.c_int),
        "rbg_build_pmh_sketches": ([vp, P(Params), C.c_char_p, i64p, C.c_int64,
                                    P(C.c_uint64), P(C.c_double)], C.c_int),
        "rbg_pmh_compare": ([vp, C.c_int32, C.c_int32, C.c_int32, vp, C.c_int64, vp,
                             C.c_int64, P(C.c_double)], C.c_int),
        "rbg_pmh_merge_registers": ([vp, P(C.c_double), P(C.c_double), C.c_int64, C.c_int32,
                                     P(C.c_double)], C.c_int),
        "rbg_pack_win16": ([vp, P(C.c_uint32), C.c_int64, P(C.c_uint16)], C.c_int),
        "rbg_estimate_pmh_baseline": ([vp, P(Params), vp, C.c_int32, C.c_int64,
                                       P(C.c_double)], C.c_int),
        "rbg_build_graph": ([vp, P(Params), P(C.c_uint32), C.c_int64, P(C.c_float),
                             C.c_int32, P(Graph)], C.c_int),
        "rbg_bin_graph": ([vp, P(Params), C.c_char_p, i64p, C.c_int64, P(C.c_float),
                           C.c_int32, P(Graph)], C.c_int),
        "rbg_bin_graph_sharded": ([vp, P(Params), P(Shard), C.c_char_p, i64p, C.c_int64,
                                   P(C.c_float), C.c_int32, P(Graph)], C.c_int),
        "rbg_stage": ([vp, C.c_char_p, i64p, C.c_int64, P(C.c_float), C.c_int32], C.c_int),
        "rbg_run_resident": ([vp, P(Params), P(Timing)], C.c_int),
        "rbg_fetch_graph": ([vp, P(Graph)], C.c_int),
        "rbg_free_graph": ([P(Graph)], C.c_int),
        "rbg_pmh_stream_tables": ([C.c_int32, C.c_int32, C.c_uint64, C.c_int32,
                                   P(C.c_int32), P(C.c_int32), P(C.c_double),
                                   P(C.c_uint32)], C.c_int),
        "rbg_bin_batch": ([vp, P(Params), P(Assembly), C.c_int32, P(Graph), P(BatchStats)],
                          C.c_int),
        "rbg_parse_fasta": ([vp, C.c_char_p, C.c_int64, C.c_int64, C.c_int64, P(Fasta)], C.c_int),
        "rbg_free_fasta": ([P(Fasta)], C.c_int),
        "rbg_bin_fasta": ([vp, P(Params), C.c_char_p, C.c_int64, C.c_int64, P(C.c_float),
                           C.c_int32, P(Graph)], C.c_int),
        "rbg_server_create": ([P(ServerConfig), P(Params), P(vp)], C.c_int),
        "rbg_server_submit": ([vp, P(Assembly), P(C.c_int64)], C.c_int),
        "rbg_server_wait": ([vp, C.c_int64, C.c_double, P(Graph), P(RequestStats)], C.c_int),
        "rbg_server_last_error": ([vp], C.c_char_p),
        "rbg_server_destroy": ([vp], C.c_int),
        "rbg_write_cache": ([C.c_char_p, P(CacheState)], C.c_int),
        "rbg_read_cache": ([C.c_char_p, P(CacheState)], C.c_int),
        "rbg_free_cache": ([P(CacheState)], C.c_int),
        "rbg_build_pmh_winners_noalloc": ([P(Params), vp, vp, C.c_int64, C.c_int64, vp, vp,
                                           C.c_char_p, C.c_size_t], C.c_int),
        "rbg_default_lpa_params": ([P(LpaParams)], C.c_int),
        "rbg_label_propagation": ([vp, P(LpaParams), C.c_int64, C.c_int64, P(C.c_uint32),
                                   P(C.c_uint32), P(C.c_float), P(C.c_uint32), P(LpaStats)],
                                  C.c_int),
        "rbg_label_propagation_resident": ([vp, P(LpaParams), P(C.c_uint32), P(LpaStats)],
                                           C.c_int),
        "rbg_default_depth_params": ([P(DepthParams)], C.c_int),
        "rbg_bam_depth": ([vp, P(C.c_char_p), C.c_int32, P(DepthParams), P(DepthMatrix)], C.c_int),
        "rbg_bam_depth_mem": ([vp, P(C.c_void_p), i64p, C.c_int32, P(DepthParams),
                               P(DepthMatrix)], C.c_int),
        "rbg_free_depth_matrix": ([P(DepthMatrix)], C.c_int),
        "rbg_depth_tsv": ([P(DepthMatrix), P(C.c_char_p), C.c_int32, P(DepthParams), C.c_int32,
                           P(C.c_void_p), i64p], C.c_int),
        "rbg_free_tsv": ([C.c_void_p], C.c_int),
        "rbg_depth_accumulate": ([vp, C.c_void_p, C.c_int64, P(C.c_uint32), C.c_int32,
                                  P(DepthParams), P(C.c_uint64), P(C.c_uint64), P(C.c_int32)],
                                 C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes, f.restype = args, res
    _lib = L
    return L


def exported_symbols():
    """Entry points declared in include/rabbitbin_b200.h."""
    hdr = os.path.join(os.path.dirname(_HERE), "include", "rabbitbin_b200.h")
    import re
    return sorted(set(re.findall(r"\b(rbg_[a-z0-9_]+)\s*\(", open(hdr).read())))


def default_depth_params(**kw):
    """rbg_default_depth_params with fields overridden by keyword."""
    p = DepthParams()
    lib().rbg_default_depth_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def default_params(**kw):
    p = Params()
    lib().rbg_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def stream_tables(k=4, m=500, pmh_seed=42, fp_contract=1):
    """(canonical codes, U [E, m] float64, W32 [E, m] uint32) of one configuration."""
    L = lib()
    ne = C.c_int32()
    rc = L.rbg_pmh_stream_tables(k, m, pmh_seed, fp_contract, C.byref(ne), None, None, None)
    if rc != RBG_OK:
        raise RbgError(rc, "stream tables")
    E = ne.value
    codes = np.zeros(E, np.int32)
    U = np.zeros((E, m), np.float64)
    W = np.zeros((E, m), np.uint32)
    rc = L.rbg_pmh_stream_tables(k, m, pmh_seed, fp_contract, C.byref(ne), _p(codes, C.c_int32),
                                 _p(U, C.c_double), _p(W, C.c_uint32))
    if rc != RBG_OK:
        raise RbgError(rc, "stream tables")
    return codes, U, W


class _GraphMem:
    """Owns one rbg_graph's library-allocated arrays; frees them when the
    last array viewing them is gone."""

    def __init__(self, L, g):
        self._L, self.g = L, g

    def __del__(self):
        try:
            self._L.rbg_free_graph(C.byref(self.g))
        except Exception:
            pass


class _View:
    """Array interface over library memory, keeping its owner alive."""

    def __init__(self, owner, addr, n, typestr):
        self.owner = owner
        self.__array_interface__ = {"shape": (n,), "typestr": typestr,
                                    "data": (addr, False), "version": 3}


def _graph_dict(L, g):
    """The graph's arrays as numpy views of the library's buffers (no copy);
    the buffers are released with rbg_free_graph when the views are gone."""
    ne = g.n_edges
    owner = _GraphMem(L, g)

    def view(ptr, typestr, dt):
        if ne == 0:
            return np.zeros(0, dt)
        return np.asarray(_View(owner, C.cast(ptr, C.c_void_p).value, ne, typestr))

    return dict(src=view(g.from_, "<u4", np.uint32), dst=view(g.to, "<u4", np.uint32),
                scomp=view(g.scomp, "<f4", np.float32), score=view(g.score, "<f4", np.float32),
                b0=g.b0, sim_cutoff=g.sim_cutoff, path=g.path)


class Context:
    """One device context (stream + device buffers), like the reference's
    per-thread sketch pool but on a GPU."""

    def __init__(self, device=0):
        self._L = lib()
        h = C.c_void_p()
        rc = self._L.rbg_create(device, C.byref(h))
        if rc != RBG_OK:
            raise RbgError(rc, f"cannot create a context on device {device}")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.rbg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != RBG_OK:
            raise RbgError(rc, f"{what}: {self._L.rbg_last_error(self._h).decode()}")

    @property
    def stream(self):
        return self._L.rbg_stream(self._h)

    def build_pmh_winners(self, seqcat, offsets, params=None):
        p = params or default_params()
        offs = np.ascontiguousarray(offsets, np.int64)
        n = len(offs) - 1
        out = np.zeros((n, p.m), np.uint32)
        self._check(self._L.rbg_build_pmh_winners(self._h, C.byref(p), seqcat, _p(offs, C.c_int64),
                                                  n, _p(out, C.c_uint32)), "build_pmh_winners")
        return out

    def build_pmh_sketches(self, seqcat, offsets, params=None):
        """(winners64 [n, m] uint64, registers [n, m] float64) of every contig's
        ProbMinHash4 sketch (rbg_build_pmh_sketches)."""
        p = params or default_params()
        offs = np.ascontiguousarray(offsets, np.int64)
        n = len(offs) - 1
        w = np.zeros((n, p.m), np.uint64)
        r = np.zeros((n, p.m), np.float64)
        self._check(self._L.rbg_build_pmh_sketches(self._h, C.byref(p), seqcat,
                                                   _p(offs, C.c_int64), n, _p(w, C.c_uint64),
                                                   _p(r, C.c_double)), "build_pmh_sketches")
        return w, r

    PMH_METRICS = {"jaccard_weighted": 0, "jaccard": 1, "distance": 2, "ani": 3}

    def pmh_compare(self, metric, A, B, kmer_size=4):
        """out[i, j] = metric(A_i, B_j) (rbg_pmh_compare); A, B: winner rows
        (uint64) for jaccard_weighted, register rows (float64) otherwise."""
        code = self.PMH_METRICS[metric]
        dt = np.uint64 if code == 0 else np.float64
        A = np.ascontiguousarray(A, dt)
        B = np.ascontiguousarray(B, dt)
        out = np.zeros((A.shape[0], B.shape[0]), np.float64)
        self._check(self._L.rbg_pmh_compare(self._h, code, A.shape[1], kmer_size,
                                            A.ctypes.data, A.shape[0], B.ctypes.data,
                                            B.shape[0], _p(out, C.c_double)), "pmh_compare")
        return out

    def pmh_merge_registers(self, A, B):
        A = np.ascontiguousarray(A, np.float64)
        B = np.ascontiguousarray(B, np.float64)
        out = np.zeros_like(A)
        self._check(self._L.rbg_pmh_merge_registers(self._h, _p(A, C.c_double), _p(B, C.c_double),
                                                    A.shape[0], A.shape[1], _p(out, C.c_double)),
                    "pmh_merge_registers")
        return out

    def build_oph_signature(self, seqcat, offsets, params):
        """One-permutation MinHash bucket values [n, m] (uint8; params.oph_k > 0)."""
        offs = np.ascontiguousarray(offsets, np.int64)
        n = len(offs) - 1
        out = np.zeros((n, params.m), np.uint8)
        self._check(self._L.rbg_build_oph_signature(self._h, C.byref(params), seqcat,
                                                    _p(offs, C.c_int64), n, _p(out, C.c_uint8)),
                    "build_oph_signature")
        return out

    def pack_win16(self, w32):
        w = np.ascontiguousarray(w32, np.uint32)
        out = np.zeros(w.shape, np.uint16)
        self._check(self._L.rbg_pack_win16(self._h, _p(w, C.c_uint32), w.size, _p(out, C.c_uint16)),
                    "pack_win16")
        return out

    def estimate_pmh_baseline(self, winners, params=None):
        p = params or default_params()
        w = np.ascontiguousarray(winners)
        bits = 16 if w.dtype == np.uint16 else 32
        b0 = C.c_double()
        self._check(self._L.rbg_estimate_pmh_baseline(self._h, C.byref(p), w.ctypes.data, bits,
                                                      w.shape[0], C.byref(b0)), "estimate_pmh_baseline")
        return b0.value

    def _graph_call(self, fn, *args):
        g = Graph()
        self._check(fn(*args, C.byref(g)), fn.__name__)
        return _graph_dict(self._L, g)

    def build_graph(self, winners32, depth, params=None):
        p = params or default_params()
        w = np.ascontiguousarray(winners32, np.uint32)
        n = w.shape[0]
        d = np.ascontiguousarray(depth, np.float32).reshape(n, -1)
        return self._graph_call(self._L.rbg_build_graph, self._h, C.byref(p), _p(w, C.c_uint32), n,
                                _p(d, C.c_float), d.shape[1])

    def bin_graph(self, seqcat, offsets, depth, params=None):
        p = params or default_params()
        offs = np.ascontiguousarray(offsets, np.int64)
        n = len(offs) - 1
        d = np.ascontiguousarray(depth, np.float32).reshape(n, -1)
        return self._graph_call(self._L.rbg_bin_graph, self._h, C.byref(p), seqcat,
                                _p(offs, C.c_int64), n, _p(d, C.c_float), d.shape[1])

    def bin_graph_sharded(self, seqcat, offsets, depth, rank, world, allgather,
                          device_buffers=False, params=None):
        """rbg_bin_graph_sharded: this rank's contigs (a contiguous part of the
        assembly, ranks in order); `allgather(send_ptr, recv_ptr, nbytes)`
        gathers nbytes from every rank (see rabbitbin_b200.shard).  Returns the
        edges whose source is one of this rank's contigs, with global ids."""
        p = params or default_params()
        offs = np.ascontiguousarray(offsets, np.int64)
        n = len(offs) - 1
        dep = np.asarray(depth, np.float32)
        S = dep.shape[1] if dep.ndim == 2 else (dep.size // n if n else 0)
        d = np.ascontiguousarray(dep.reshape(n, S))

        def call(send, recv, nbytes, user):
            try:
                allgather(send, recv, nbytes)
                return 0
            except Exception:               # a Python exception must not look like success
                return 1
        fn = ALLGATHER_FN(call)
        sh = Shard(rank, world, 1 if device_buffers else 0, 0, fn, None)
        return self._graph_call(self._L.rbg_bin_graph_sharded, self._h, C.byref(p), C.byref(sh),
                                seqcat, _p(offs, C.c_int64), n, _p(d, C.c_float), d.shape[1])

    def stage(self, seqcat, offsets, depth):
        offs = np.ascontiguousarray(offsets, np.int64)
        n = len(offs) - 1
        d = np.ascontiguousarray(depth, np.float32).reshape(n, -1)
        self._check(self._L.rbg_stage(self._h, seqcat, _p(offs, C.c_int64), n, _p(d, C.c_float),
                                      d.shape[1]), "stage")

    def run_resident(self, params=None):
        p = params or default_params()
        t = Timing()
        self._check(self._L.rbg_run_resident(self._h, C.byref(p), C.byref(t)), "run_resident")
        return t.as_dict()

    def fetch_graph(self):
        return self._graph_call(self._L.rbg_fetch_graph, self._h)

    @staticmethod
    def _lpa_params(seed, rule, synchronous, node_order, max_rounds):
        lp = LpaParams()
        lib().rbg_default_lpa_params(C.byref(lp))
        if seed is not None:
            lp.seed = int(seed)
        if rule is not None:
            lp.score_rule = LPA_RULES[rule] if isinstance(rule, str) else int(rule)
        if synchronous is not None:
            lp.synchronous = int(bool(synchronous))
        lp.max_rounds = int(max_rounds)
        order = None
        if node_order is not None:
            order = np.ascontiguousarray(node_order, np.uint32)
            lp.node_order = order.ctypes.data
        return lp, order

    def label_propagation(self, n_nodes, src, dst, score, seed=None, rule=None,
                          synchronous=None, node_order=None, max_rounds=0):
        """cluster_by_propagation on an edge list (rbg_label_propagation):
        (membership uint32[n_nodes], stats dict).  rule: a RABBIT_LPA_SCORE
        name or RBG_LPA_* value; None takes the environment, as the reference."""
        lp, order = self._lpa_params(seed, rule, synchronous, node_order, max_rounds)
        f = np.ascontiguousarray(src, np.uint32)
        t = np.ascontiguousarray(dst, np.uint32)
        w = np.ascontiguousarray(score, np.float32)
        out = np.zeros(int(n_nodes), np.uint32)
        st = LpaStats()
        self._check(self._L.rbg_label_propagation(
            self._h, C.byref(lp), int(n_nodes), len(f), _p(f, C.c_uint32), _p(t, C.c_uint32),
            _p(w, C.c_float), _p(out, C.c_uint32), C.byref(st)), "label_propagation")
        del order
        return out, st.as_dict()

    def label_propagation_resident(self, n_nodes, seed=None, rule=None, synchronous=None,
                                   node_order=None, max_rounds=0):
        """Label propagation on the graph of the last bin_graph / run_resident
        call, still on the device (rbg_label_propagation_resident)."""
        lp, order = self._lpa_params(seed, rule, synchronous, node_order, max_rounds)
        out = np.zeros(int(n_nodes), np.uint32)
        st = LpaStats()
        self._check(self._L.rbg_label_propagation_resident(
            self._h, C.byref(lp), _p(out, C.c_uint32), C.byref(st)),
            "label_propagation_resident")
        del order
        return out, st.as_dict()

    def bam_depth(self, bams, tsv_names=None, tsv_variance=False, **kw):
        """Depth matrix of BAM files (rbg_bam_depth_mem for bytes, rbg_bam_depth
        for paths): dict with names, lens, tid, means [rows, cols], sums
        [cols, n_targets], avg_read, records and timings; with tsv_names (the
        BAMs' file names) also "tsv", the depth table (rbg_depth_tsv).
        Keywords set rbg_depth_params fields."""
        p = default_depth_params(**kw)
        m = DepthMatrix()
        n = len(bams)
        if all(isinstance(b, (bytes, bytearray, memoryview, np.ndarray)) for b in bams):
            # the callers' buffers themselves, without a copy
            keep = [np.frombuffer(b, np.uint8) for b in bams]
            ptrs = (C.c_void_p * n)(*[k.ctypes.data if len(k) else None for k in keep])
            sizes = np.asarray([len(b) for b in bams], np.int64)
            rc = self._L.rbg_bam_depth_mem(self._h, ptrs, _p(sizes, C.c_int64), n, C.byref(p),
                                           C.byref(m))
        else:
            keep = [os.fsencode(b) for b in bams]
            ptrs = (C.c_char_p * n)(*keep)
            rc = self._L.rbg_bam_depth(self._h, ptrs, n, C.byref(p), C.byref(m))
        self._check(rc, "bam_depth")
        try:
            tsv = None
            if tsv_names is not None:
                nm = (C.c_char_p * n)(*[os.fsencode(x) for x in tsv_names])
                buf, ln = C.c_void_p(), C.c_int64()
                st = self._L.rbg_depth_tsv(C.byref(m), nm, n, C.byref(p), int(bool(tsv_variance)),
                                           C.byref(buf), C.byref(ln))
                if st != RBG_OK:
                    raise RbgError(st, "depth_tsv")
                tsv = C.string_at(buf, ln.value)
                self._L.rbg_free_tsv(buf)
            nr, nc, nt = int(m.n_rows), int(m.n_cols), int(m.n_targets)
            names = []
            if nr:
                # one read of the NUL-terminated names block
                off = np.ctypeslib.as_array(m.name_off, (nr,))
                last = int(off[-1])
                tail = C.string_at(m.names + last)
                blob = C.string_at(m.names, last + len(tail) + 1)
                names = blob[:-1].decode().split("\0")
            out = {
                "names": names,
                "tid": np.ctypeslib.as_array(m.tid, (nr,)).copy() if nr else np.zeros(0, np.int32),
                "lens": np.ctypeslib.as_array(m.lens, (nr,)).copy() if nr else np.zeros(0, np.int32),
                "means": (np.ctypeslib.as_array(m.means, (nr * nc,)).reshape(nr, nc).copy()
                          if nr * nc else np.zeros((nr, nc), np.float32)),
                "sums": (np.ctypeslib.as_array(m.sums, (nc * nt,)).reshape(nc, nt).copy()
                         if nc * nt else np.zeros((nc, nt), np.uint64)),
                "avg_read": np.ctypeslib.as_array(m.avg_read, (n,)).copy(),
                "records": int(m.records), "compressed_bytes": int(m.compressed_bytes),
                "decompressed_bytes": int(m.decompressed_bytes),
                "inflate_ms": float(m.inflate_ms), "total_ms": float(m.total_ms),
                "kernel_ms": float(m.kernel_ms), "device_bams": int(m.device_bams),
                "tsv": tsv,
            }
        finally:
            self._L.rbg_free_depth_matrix(C.byref(m))
        return out

    def depth_accumulate(self, records, target_len, **kw):
        """One sample's depth sums from decompressed records
        (rbg_depth_accumulate): (sums, sums with MAPQ >= dual_map_qual, avg_read)."""
        p = default_depth_params(**kw)
        rec = np.frombuffer(bytes(records), np.uint8) if len(records) else np.zeros(1, np.uint8)
        tl = np.ascontiguousarray(target_len, np.uint32)
        nt = len(tl)
        d = np.zeros(max(nt, 1), np.uint64)
        du = np.zeros(max(nt, 1), np.uint64)
        avg = C.c_int32(0)
        self._check(self._L.rbg_depth_accumulate(
            self._h, rec.ctypes.data, len(records), _p(tl, C.c_uint32), nt, C.byref(p),
            _p(d, C.c_uint64), _p(du, C.c_uint64), C.byref(avg)), "depth_accumulate")
        return d[:nt], du[:nt], int(avg.value)

    def parse_fasta(self, data, min_contig=2500, min_small_contig=1000):
        """Device FASTA parse (rbg_parse_fasta) of the bytes `data`:
        {num_seqs, large: (seqcat, offsets, names), small: (...)}."""
        f = Fasta()
        self._check(self._L.rbg_parse_fasta(self._h, data, len(data), min_contig,
                                            min_small_contig, C.byref(f)), "parse_fasta")
        try:
            out = {"num_seqs": f.num_seqs}
            for tag, n, seq, off, ns, nl in (
                    ("large", f.n_large, f.large_seq, f.large_off, f.large_name_start,
                     f.large_name_len),
                    ("small", f.n_small, f.small_seq, f.small_off, f.small_name_start,
                     f.small_name_len)):
                offs = np.ctypeslib.as_array(off, (n + 1,)).copy()
                seqcat = C.string_at(seq, int(offs[-1])) if offs[-1] else b""
                names = [data[ns[i]:ns[i] + nl[i]] for i in range(n)]
                out[tag] = (seqcat, offs, names)
            return out
        finally:
            self._L.rbg_free_fasta(C.byref(f))

    def bin_fasta(self, data, depth, min_contig=2500, params=None, nbytes=None):
        """The hot path from FASTA bytes (rbg_bin_fasta); depth rows are the
        large contigs in file order.  `data` is bytes, or a char pointer with
        `nbytes` (e.g. pinned host memory)."""
        p = params or default_params()
        d = np.ascontiguousarray(depth, np.float32)
        S = d.shape[1] if d.ndim == 2 else 0
        n = len(data) if nbytes is None else nbytes
        return self._graph_call(self._L.rbg_bin_fasta, self._h, C.byref(p), data, n,
                                min_contig, _p(d, C.c_float) if d.size else None, S)

    def bin_batch(self, assemblies, params=None):
        """Graphs of many assemblies in one call (rbg_bin_batch).

        `assemblies`: sequence of (seqcat, offsets, depth) or
        (seqcat, offsets, depth, params); depth is n x S (S may be 0).
        Returns (list of graph dicts in input order, stats dict)."""
        dflt = params or default_params()
        nb = len(assemblies)
        arr = (Assembly * max(nb, 1))()
        keep = []
        for i, a in enumerate(assemblies):
            seq, offs, depth = a[0], a[1], a[2]
            p = a[3] if len(a) > 3 and a[3] is not None else None
            offs = np.ascontiguousarray(offs, np.int64)
            n = len(offs) - 1
            dep = np.ascontiguousarray(depth, np.float32)
            S = dep.shape[1] if dep.ndim == 2 else (dep.size // n if n > 0 else 0)
            d = dep.reshape(n, S)
            keep += [seq, offs, d, p]
            arr[i].seqcat = seq
            arr[i].offsets = _p(offs, C.c_int64)
            arr[i].n = n
            arr[i].depth = _p(d, C.c_float) if d.size else None
            arr[i].S = S
            arr[i].params = C.pointer(p) if p is not None else None
        outs = (Graph * max(nb, 1))()
        st = BatchStats()
        self._check(self._L.rbg_bin_batch(self._h, C.byref(dflt), arr, nb, outs, C.byref(st)),
                    "bin_batch")
        graphs = []
        for i in range(nb):
            g = Graph()
            C.pointer(g)[0] = outs[i]
            graphs.append(_graph_dict(self._L, g))
        return graphs, st.as_dict()


class Server:
    """Request loop of the serving form (rbg_server_*): submit assemblies as
    they arrive, wait for their graphs.  Arrays passed to submit are kept
    alive here until their request has been waited for."""

    def __init__(self, device=0, workers=0, hbm_budget=0, max_batch=64, plain=False,
                 params=None, max_batch_pairs=0, small_pairs=0):
        self._L = lib()
        cfg = ServerConfig(device, workers, int(hbm_budget), max_batch, 1 if plain else 0,
                           int(max_batch_pairs), int(small_pairs))
        h = C.c_void_p()
        p = params or default_params()
        rc = self._L.rbg_server_create(C.byref(cfg), C.byref(p), C.byref(h))
        if rc != RBG_OK:
            raise RbgError(rc, "cannot create the server")
        self._h = h
        self._keep = {}

    def _check(self, rc, what):
        if rc != RBG_OK:
            raise RbgError(rc, f"{what}: {self._L.rbg_server_last_error(self._h).decode()}")

    def submit(self, seqcat, offsets, depth, params=None):
        offs = np.ascontiguousarray(offsets, np.int64)
        n = len(offs) - 1
        dep = np.ascontiguousarray(depth, np.float32)
        S = dep.shape[1] if dep.ndim == 2 else (dep.size // n if n > 0 else 0)
        d = dep.reshape(n, S)
        a = Assembly()
        a.seqcat = seqcat
        a.offsets = _p(offs, C.c_int64)
        a.n = n
        a.depth = _p(d, C.c_float) if d.size else None
        a.S = S
        a.params = C.pointer(params) if params is not None else None
        rid = C.c_int64()
        self._check(self._L.rbg_server_submit(self._h, C.byref(a), C.byref(rid)), "submit")
        self._keep[rid.value] = (seqcat, offs, d, params)
        return rid.value

    def wait(self, rid, timeout=-1.0):
        """(graph dict, stats dict); raises RbgError (code -5) on timeout."""
        g = Graph()
        st = RequestStats()
        rc = self._L.rbg_server_wait(self._h, rid, float(timeout), C.byref(g), C.byref(st))
        if rc == -5:
            raise RbgError(rc, f"request {rid} not finished")
        self._keep.pop(rid, None)
        self._check(rc, f"request {rid}")
        return _graph_dict(self._L, g), st.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            self._L.rbg_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
