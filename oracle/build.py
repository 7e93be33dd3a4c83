"""Build recipe for the oracle libraries (test infrastructure only).

Two host libraries come out of this script:

* ``oracle/_build/librboracle.so`` — the CPU restatement in ``oracle/rb_oracle.cpp``
  (committed source, always buildable).
* ``oracle/_ref/librbref.so`` — RabbitBin's own hot-path code, compiled from the
  reference tree where it lies.  ``src/probmh.cpp`` is compiled whole; the
  functions that live inside the (unbuildable, Boost/libdeflate-dependent)
  ``src/rabbitbin.cpp`` TU and the graph module ``src/impl/rb_graph.cpp`` are cut
  out by line range into ``oracle/_ref/frag/`` at build time and #included by
  ``oracle/ref_shim.cpp``.  Nothing from the reference tree is committed; the
  ``_ref`` folder is git-ignored and travels to the GPU box prebuilt.

Both are compiled with the reference's release flags
(``src/CMakeLists.txt:211-253``: ``-O3 -march=native -funroll-loops -fopenmp``),
with ``-march=x86-64-v4`` (AVX-512F/BW/DQ/VL) in place of ``native`` so the
prebuilt library runs on any AVX-512 host and follows the AVX-512 code paths of
the reference on every machine.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference tree: RABBITBIN_REFERENCE, else a checkout named "reference"
# beside this repository (absent on machines that only run the prebuilt files)
REF = os.environ.get("RABBITBIN_REFERENCE") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")
REF_SRC = os.path.join(REF, "src")
FLAGS = ["-std=c++17", "-O3", "-march=x86-64-v4", "-funroll-loops", "-fopenmp",
         "-fPIC", "-shared", "-w"]

# (fragment name, reference file, first line, last line)
FRAGMENTS = [
    ("frag_random_unique.inc", "rabbitbin.h", 330, 341),
    ("frag_compare_edge.inc", "rabbitbin.h", 418, 429),
    ("frag_fold16.inc", "rabbitbin.cpp", 249, 253),
    ("frag_depth_terms.inc", "rabbitbin.cpp", 685, 970),
    ("frag_jaccard_raw.inc", "rabbitbin.cpp", 1031, 1135),
    ("frag_pmh_sim.inc", "rabbitbin.cpp", 1194, 1426),
    ("frag_build_winners.inc", "rabbitbin.cpp", 1436, 1589),
    ("frag_contig_rec.inc", "rabbitbin.cpp", 1876, 1888),
    ("frag_parse_fasta.inc", "rabbitbin.cpp", 1890, 2248),
    ("frag_anynz.inc", "impl/rb_abundance.cpp", 94, 114),
    ("frag_graph_allpairs.inc", "impl/rb_graph.cpp", 7, 72),
    ("frag_graph_index.inc", "impl/rb_graph.cpp", 199, 383),
    ("frag_calib_converge.inc", "impl/rb_graph.cpp", 390, 415),
    ("frag_fused_graph.inc", "impl/rb_graph.cpp", 489, 1356),
    ("frag_calibrate.inc", "impl/rb_graph.cpp", 1362, 1384),
    ("frag_calibrate_fused.inc", "impl/rb_graph.cpp", 1386, 1438),
    ("frag_cache.inc", "impl/rb_cache.cpp", 26, 319),
    ("frag_lpa_rules.inc", "impl/rb_cluster.cpp", 3, 93),
    ("frag_lpa.inc", "impl/rb_cluster.cpp", 336, 740),
    ("frag_incidence.inc", "rabbitbin.cpp", 5600, 5622),
    ("frag_node_order.inc", "rabbitbin.cpp", 5643, 5645),
    ("frag_bam_chooser.inc", "BamUtils.h", 275, 318),
    ("frag_checkread.inc", "CheckRead.hpp", 20, 276),
    ("frag_thread_blocker.inc", "rabbit_depth.h", 48, 66),
    ("frag_depth_counts.inc", "rabbit_depth.h", 70, 162),
    ("frag_read_stats.inc", "rabbit_depth.h", 181, 376),
    ("frag_caldepth.inc", "rabbit_depth.h", 601, 887),
    ("frag_depth_column.inc", "rabbit_depth_fuse.h", 65, 68),
    ("frag_depth_accumulate.inc", "rabbit_depth.cpp", 1615, 1685),
    ("frag_variance_type.inc", "rabbit_depth.h", 164, 176),
    ("frag_depth_basename.inc", "rabbit_depth.cpp", 114, 123),
    ("frag_depth_table.inc", "rabbit_depth.cpp", 125, 313),
]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_oracle():
    """Compile the restatement oracle into oracle/_build/librboracle.so."""
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "librboracle.so")
    src = os.path.join(HERE, "rb_oracle.cpp")
    if _stale(out, [src, __file__]):
        _run(["g++"] + FLAGS + [src, "-o", out])
    return out


def build_ref():
    """Compile the reference harness into oracle/_ref/librbref.so.

    Returns the path, or None when the reference tree is absent (GPU box: the
    prebuilt library travels with the snapshot instead)."""
    out_dir = os.path.join(HERE, "_ref")
    out = os.path.join(out_dir, "librbref.so")
    if not os.path.isdir(REF_SRC):
        return out if os.path.exists(out) else None
    frag_dir = os.path.join(out_dir, "frag")
    os.makedirs(frag_dir, exist_ok=True)
    for name, rel, a, b in FRAGMENTS:
        with open(os.path.join(REF_SRC, rel), encoding="utf-8") as f:
            lines = f.readlines()
        text = "".join(lines[a - 1:b])
        path = os.path.join(frag_dir, name)
        if not os.path.exists(path) or open(path, encoding="utf-8").read() != text:
            with open(path, "w", encoding="utf-8") as f:
                f.write(text)
    shim = os.path.join(HERE, "ref_shim.cpp")
    cache_shim = os.path.join(HERE, "ref_cache_shim.cpp")
    lpa_shim = os.path.join(HERE, "ref_lpa_shim.cpp")
    depth_shim = os.path.join(HERE, "ref_depth_shim.cpp")
    deps = [shim, cache_shim, lpa_shim, depth_shim, os.path.join(HERE, "htslib_shim.h"), __file__,
            os.path.join(REF_SRC, "probmh.cpp")]
    if _stale(out, deps):
        _run(["g++"] + FLAGS + ["-I", frag_dir, "-I", REF_SRC, shim, cache_shim, lpa_shim,
                                os.path.join(REF_SRC, "probmh.cpp"), "-o", out])
    # the depth harness includes the reference's BamUtils.h fragments against the
    # htslib stand-in; it is a separate library so that those headers' names do
    # not meet the graph harness's
    dout = os.path.join(out_dir, "librbref_depth.so")
    if _stale(dout, deps):
        _run(["g++"] + FLAGS + ["-I", frag_dir, "-I", HERE, depth_shim, "-o", dout])
    return out


if __name__ == "__main__":
    print(build_oracle())
    print(build_ref())
