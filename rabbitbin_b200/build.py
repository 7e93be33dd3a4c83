"""Build librabbitbin_b200.so in-tree (sm_100a CUDA kernels + C++ host engine).

    python -m rabbitbin_b200.build

nvcc cross-compiles for sm_100a without a GPU.  Kernels are compiled with
-fmad=false (explicit __fma*_rn where the reference fuses); host C++ with
-ffp-contract=off for the same reason.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "librabbitbin_b200.so")
BUILD = os.path.join(HERE, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SRCS = ["kernels_sketch.cu", "kernels_graph.cu", "kernels_allpairs.cu", "kernels_onehot.cu",
           "kernels_onehot_mma.cu", "kernels_sym_tc5.cu", "kernels_pmh_query.cu", "kernels_index.cu",
           "kernels_util.cu",
           "noalloc.cu", "kernels_fasta.cu", "kernels_lpa.cu", "kernels_depth.cu"]
CPP_SRCS = ["pmh_streams.cpp", "calib.cpp", "engine.cpp", "batch.cpp", "server.cpp", "fasta.cpp",
            "cache.cpp", "host_pack.cpp", "lpa.cpp", "bam.cpp"]
HEADERS = ["rbg_internal.h", "engine_internal.h", "select_topk.cuh", "tc05.cuh", "ddmath.cuh",
           "depth_record.cuh",
           "../../include/rabbitbin_b200.h", "gen_zig_tables.py"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build failed: " + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    zig = os.path.join(CSRC, "zig_tables.inc")
    gen = os.path.join(CSRC, "gen_zig_tables.py")
    if _newer(zig, [gen]):
        _run([sys.executable, gen, zig])
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [zig]
    objs = []
    for src in CU_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _newer(o, [s, __file__] + hdrs) or ptxas_info:
            cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-fmad=false", "-std=c++17",
                                   "-Xcompiler", "-fPIC", "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            log = _run(cmd)
            if verbose or ptxas_info:
                print(log)
        objs.append(o)
    for src in CPP_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if _newer(o, [s, __file__] + hdrs):
            _run(["g++", "-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-march=x86-64-v2",
                  "-I", os.path.join(CUDA, "include"), "-c", s, "-o", o])
        objs.append(o)
    if _newer(OUT, objs):
        tmp = OUT + ".tmp"
        lib64 = os.path.join(CUDA, "lib64")
        _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs +
             ["-cudart", "static", "-L" + lib64, "-Xlinker", "-rpath=" + lib64, "-lz"])
        shutil.move(tmp, OUT)
    return OUT


def build_synth():
    """The synthetic-assembly chain and BAM generators (host C, OpenMP)."""
    srcs = [os.path.join(CSRC, "synth_chain.c"), os.path.join(CSRC, "synth_bam.c")]
    out = os.path.join(HERE, "libsynth_chain.so")
    if _newer(out, srcs):
        _run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared"] + srcs + ["-o", out, "-lz", "-lm"])
    return out


if __name__ == "__main__":
    build_synth()
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
