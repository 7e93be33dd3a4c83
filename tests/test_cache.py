"""RBCACHE1 files (rbg_write_cache / rbg_read_cache) against RabbitBin's own
rb_write_cache / rb_load_cache (src/impl/rb_cache.cpp:103-319), compiled in
the reference harness.  Host-only: no device is needed.

* the product and the reference write byte-identical files for one state;
* each reads the other's file back to the same state;
* files of versions 1 and 2 (size_t endpoints; version 1 without the SNV
  block), written here by a small independent writer of the documented
  layout, read the same in both programs;
* truncated or foreign files are rejected by both.
"""
import struct

import numpy as np
import pytest

import oracle
from rabbitbin_b200 import api


def _state(seed, snv=True, depth=True):
    rng = np.random.default_rng(seed)
    nl, ns, S = 57, 13, 6 if depth else 0
    ne = 211
    st = {
        "n_large": nl, "n_small": ns, "samples": S, "seed": 1, "total_size": 123456789,
        "total_size_small": 23456, "sim_cutoff": 799.5, "b0": 0.3880000114440918,
        "min_contig": 2500, "min_small_contig": 1000, "has_depth": int(depth),
        "has_snv": int(snv),
        "large_names": [b"contig_%d" % i + b"x" * int(rng.integers(0, 9)) for i in range(nl)],
        "small_names": [b"s%d" % i for i in range(ns)] + [b""][:0],
        "large_len": rng.integers(2500, 80000, nl).astype(np.uint64),
        "small_len": rng.integers(1000, 2500, ns).astype(np.uint64),
        "depth_ranked": (rng.integers(2, 2 * S + 1, (nl, S)) / 2.0).astype(np.float32)
        if depth else np.zeros((0, 0), np.float32),
        "small_depth": rng.random((ns, S), np.float32) if depth else np.zeros((0, 0), np.float32),
        "large_means": rng.random(nl * S, np.float32) if depth else np.zeros(0, np.float32),
        "depth_raw": rng.random(nl * S, np.float32) if depth else np.zeros(0, np.float32),
        "colnorm": rng.random(S) if depth else np.zeros(0),
        "from_": rng.integers(0, nl, ne).astype(np.uint32),
        "to": rng.integers(0, nl, ne).astype(np.uint32),
        "scomp": rng.random(ne, np.float32),
    }
    if snv:
        st["snv_pi"] = rng.random(nl * S, np.float32)
        st["snv_nsnv"] = rng.integers(0, 100, nl * S).astype(np.uint32)
        st["snv_cov"] = rng.integers(0, 10000, nl * S).astype(np.uint32)
    return st


def _same(a, b, ref_read=False):
    for k in api.CACHE_SCALARS:
        if k == "has_snv" and not a[k] and not b[k]:
            continue
        if ref_read and k in ("min_contig", "min_small_contig"):
            continue        # rb_load_cache reads them and keeps neither (informational)
        assert a[k] == b[k], k
    assert a["large_names"] == b["large_names"] and a["small_names"] == b["small_names"]
    for name, dt, _ in api.CACHE_ARRAYS:
        x = np.asarray(a.get(name, np.zeros(0, dt)), dt)
        y = np.asarray(b.get(name, np.zeros(0, dt)), dt)
        if x.size == 0 and y.size == 0:
            continue
        assert np.array_equal(x.reshape(-1), y.reshape(-1)), name


@pytest.mark.parametrize("snv,depth", [(True, True), (False, True), (False, False)])
def test_files_identical_and_cross_read(ref_lib, tmp_path, snv, depth):
    st = _state(3, snv=snv, depth=depth)
    a, b = tmp_path / "ours.rbc", tmp_path / "ref.rbc"
    api.write_cache(a, st)
    oracle.ref_cache_write(b, st)
    assert a.read_bytes() == b.read_bytes()
    ours = api.read_cache(b)
    assert ours["version"] == 3
    _same(ours, st)
    _same(oracle.ref_cache_read(a), st, ref_read=True)


def _legacy_file(st, version):
    """The documented layout with size_t endpoints (versions 1 and 2)."""
    out = bytearray(b"RBCACHE1")
    pack = lambda fmt, *v: out.extend(struct.pack("<" + fmt, *v))
    pack("III", version, 4, 8)
    pack("QQQQQQ", st["n_large"], st["n_small"], st["samples"], st["seed"], st["total_size"],
         st["total_size_small"])
    pack("dd", st["sim_cutoff"], st["b0"])
    pack("QQB", st["min_contig"], st["min_small_contig"], st["has_depth"])
    for key in ("large_names", "small_names"):
        pack("Q", len(st[key]))
        for nm in st[key]:
            pack("I", len(nm))
            out.extend(nm)

    def vec(a, fmt):
        a = np.asarray(a)
        pack("Q", a.size)
        out.extend(np.ascontiguousarray(a, fmt).tobytes())
    vec(st["large_len"], "<u8")
    vec(st["small_len"], "<u8")
    for m in ("depth_ranked", "small_depth"):
        r, c = st[m].shape
        pack("QQ", r, c)
        out.extend(np.ascontiguousarray(st[m], "<f4").tobytes())
    vec(st["large_means"], "<f4")
    vec(st["depth_raw"], "<f4")
    vec(st["colnorm"], "<f8")
    vec(st["from_"].astype(np.uint64), "<u8")
    vec(st["to"].astype(np.uint64), "<u8")
    vec(st["scomp"], "<f4")
    if version >= 2:
        pack("B", 1 if st.get("has_snv") else 0)
        if st.get("has_snv"):
            vec(st["snv_pi"], "<f4")
            vec(st["snv_nsnv"], "<u4")
            vec(st["snv_cov"], "<u4")
    return bytes(out)


@pytest.mark.parametrize("version", [1, 2])
def test_legacy_versions(ref_lib, tmp_path, version):
    st = _state(4, snv=version == 2)
    p = tmp_path / f"v{version}.rbc"
    p.write_bytes(_legacy_file(st, version))
    ours, theirs = api.read_cache(p), oracle.ref_cache_read(p)
    assert theirs is not None and ours["version"] == version
    _same(theirs, ours, ref_read=True)
    _same(ours, st if version == 2 else dict(st, has_snv=0))


def test_rejects_damaged_files(ref_lib, tmp_path):
    st = _state(5)
    good = tmp_path / "good.rbc"
    api.write_cache(good, st)
    data = good.read_bytes()
    cases = {"truncated": data[:len(data) // 2], "magic": b"RBCACHE2" + data[8:],
             "abi": data[:12] + struct.pack("<I", 8) + data[16:],
             "endpoint": None}
    # an edge endpoint past n_large
    st2 = dict(st)
    st2["to"] = st["to"].copy()
    st2["to"][3] = st["n_large"] + 5
    bad = tmp_path / "endpoint.rbc"
    api.write_cache(bad, st2)
    cases["endpoint"] = bad.read_bytes()
    for name, blob in cases.items():
        p = tmp_path / (name + ".rbc")
        p.write_bytes(blob)
        with pytest.raises(api.RbgError):
            api.read_cache(p)
        assert oracle.ref_cache_read(p) is None, name
