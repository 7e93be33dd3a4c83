"""BAM -> depth summariser on the CPU: the library's per-record rule
(rabbitbin_b200/csrc/depth_record.cuh, the code the device kernel runs,
compiled here for the host by tests/native/depth_rule_host.cpp) against the
reference's own depth_accumulate_sample (oracle/_ref/librbref_depth.so) and
against the golden sums made from it (tests/golden/depth.npz)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle
from depth_cases import CASES, PARAMS, case
from rabbitbin_b200.synth import bam_records

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def rule(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("depth_rule") / "librule.so")
    subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared",
                    os.path.join(HERE, "native", "depth_rule_host.cpp"), "-o", out], check=True)
    lib = C.CDLL(out)
    lib.host_depth_rule.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int32, C.c_float,
                                    C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p]

    def run(recs, tl, pid, edge, inc, mq, dq):
        rec = np.frombuffer(recs, np.uint8) if len(recs) else np.zeros(1, np.uint8)
        tl = np.ascontiguousarray(tl, np.uint32)
        s = np.zeros(max(len(tl), 1), np.uint64)
        su = np.zeros_like(s)
        avg = C.c_int32()
        rc = lib.host_depth_rule(rec.ctypes.data, len(recs), tl.ctypes.data, len(tl), C.c_float(pid),
                                 edge, int(inc), mq, dq, s.ctypes.data, su.ctypes.data,
                                 C.byref(avg))
        assert rc == 0
        return s[:len(tl)], su[:len(tl)], avg.value
    return run


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "depth.npz"))


@pytest.mark.parametrize("name", sorted(CASES))
def test_rule_matches_golden(rule, golden, name):
    _, _, bam = case(name)
    recs, tl, _ = bam_records(bam)
    for i, (pid, edge, inc, mq, dq) in enumerate(PARAMS):
        s, su, avg = rule(recs, tl, pid, edge, inc, mq, dq)
        assert avg == int(golden[f"{name}/{i}/avg"])
        np.testing.assert_array_equal(s, golden[f"{name}/{i}/sums"], err_msg=f"{name} params {i}")
        if dq:
            np.testing.assert_array_equal(su, golden[f"{name}/{i}/sums_u"])


def test_rule_matches_reference_random(rule):
    """Fresh seeds, checked against the reference's code itself."""
    if oracle.ref_depth() is None:
        pytest.skip("reference harness not built")
    rng = np.random.default_rng(5)
    for seed in range(6):
        lens = rng.integers(0, 6000, 60).astype(np.uint32)
        depth = rng.uniform(0.1, 30, 60)
        from rabbitbin_b200.synth import make_bam
        bam = make_bam(lens, depth, seed=100 + seed, read_len=int(rng.choice([50, 100, 150, 300])),
                       p_overhang=0.2, p_eqx=0.3, p_mixed=0.2, p_nm_off=0.2, err_mean=0.03)
        recs, tl, _ = bam_records(bam)
        pid = float(rng.choice([0.97, 0.95, 0.8]))
        edge = int(rng.choice([0, 30, 75]))
        s, _, avg = rule(recs, tl, pid, edge, False, 0, 0)
        want, wavg = oracle.depth_accumulate_ref(recs, tl, pid, edge, False, 0)
        assert avg == wavg
        np.testing.assert_array_equal(s, want)


def test_means_formula():
    sums = np.array([0, 10, 1000, 2**40, 5, 7, 9], np.uint64)
    tl = np.array([3, 151, 153, 1000, 2, 10, 152], np.uint32)
    m = oracle.depth_means(sums, tl, 75)
    assert m[0] == np.float32(0.0)                    # adj = len = 3 > 2: 0 / 3
    assert m[1] == np.float32(10 / 151)                # len <= 2 edge + 1: whole length
    assert m[2] == np.float32(1000 / 3)                # 153 - 150
    assert m[3] == 0                                   # above 1e6: cleared
    assert m[4] == 0                                   # adj <= 2
    assert m[5] == np.float32(7 / 10)
    assert m[6] == 0                                   # 152 - 150 = 2: adj <= 2


def _matrix(api_mod, sums, avg, tl, names, min_len, nb):
    """An rbg_depth_matrix as rbg_bam_depth returns it, built on the host."""
    import ctypes as C
    kept = np.nonzero(tl.astype(np.int64) >= min_len)[0].astype(np.int32)
    blob = b"".join(names[t].encode() + b"\0" for t in kept) or b"\0"
    off = np.zeros(max(len(kept), 1), np.int64)
    o = 0
    for i, t in enumerate(kept):
        off[i] = o
        o += len(names[t].encode()) + 1
    lens = tl[kept].astype(np.int32)
    sums = np.ascontiguousarray(sums, np.uint64)
    avg = np.ascontiguousarray(avg, np.int32)
    keep = [kept, blob, off, lens, sums, avg]
    m = api_mod.DepthMatrix()
    m.n_rows, m.n_cols, m.n_targets = len(kept), nb, len(tl)
    m.tid = kept.ctypes.data_as(C.POINTER(C.c_int32))
    m.lens = lens.ctypes.data_as(C.POINTER(C.c_int32))
    bbuf = C.create_string_buffer(blob, len(blob))
    keep.append(bbuf)
    m.names = C.cast(bbuf, C.c_void_p)
    m.name_off = off.ctypes.data_as(C.POINTER(C.c_int64))
    m.avg_read = avg.ctypes.data_as(C.POINTER(C.c_int32))
    m.sums = sums.ctypes.data_as(C.POINTER(C.c_uint64))
    return m, keep


def test_depth_table_matches_reference_printer():
    """rbg_depth_tsv (host formatting of the device sums) against the
    reference's own printDepthTable, byte for byte."""
    import ctypes as C
    from rabbitbin_b200 import api
    from rabbitbin_b200.synth import make_bam
    if oracle.ref_depth() is None:
        pytest.skip("reference harness not built")
    L = api.lib()
    rng = np.random.default_rng(8)
    lens, _, _ = case("edge_mix")
    names = [f"ctg_{i}" + (" some description" if i % 5 == 0 else "") +
             ("\tx" if i % 7 == 0 else "") for i in range(len(lens))]
    for nb, read_lens, seeds in ((1, [150], [200]), (3, [150, 60, 250], [200, 201, 202]),
                                 (2, [150, 100], [11, 77])):
        sums, avg = [], []
        for b in range(nb):
            bam = make_bam(lens, rng.uniform(0.1, 40, len(lens)), seed=seeds[b],
                           read_len=read_lens[b])
            recs, tl, _ = bam_records(bam)
            s, a = oracle.depth_accumulate_ref(recs, tl, 0.97, 75, False, 0)
            sums.append(s)
            avg.append(a)
        sums = np.stack(sums)
        for variance in (False, True):
            for inc, edge, min_len in ((False, 75, 1), (True, 75, 1), (False, 20, 1000),
                                       (False, 300, 1)):
                want = oracle.depth_tsv_ref(sums, avg, lens, names,
                                            [f"/data/run{b}/sample{b}.sorted.bam" for b in range(nb)],
                                            variance, inc, edge, min_len)
                m, keep = _matrix(api, sums, avg, lens, names, min_len, nb)
                p = api.default_depth_params(include_edge_bases=int(inc), max_edge_bases=edge,
                                             min_contig_length=min_len)
                bn = (C.c_char_p * nb)(*[f"/data/run{b}/sample{b}.sorted.bam".encode()
                                        for b in range(nb)])
                buf, ln = C.c_void_p(), C.c_int64()
                assert L.rbg_depth_tsv(C.byref(m), bn, nb, C.byref(p), int(variance),
                                       C.byref(buf), C.byref(ln)) == 0
                got = C.string_at(buf, ln.value)
                L.rbg_free_tsv(buf)
                assert got == want, (nb, variance, inc, edge, min_len)


def test_depth_table_large_threaded():
    """A table large enough to be formatted on several host threads (30,000
    contigs x 4 BAMs): still the reference printer's bytes."""
    import ctypes as C
    from rabbitbin_b200 import api
    if oracle.ref_depth() is None:
        pytest.skip("reference harness not built")
    L = api.lib()
    rng = np.random.default_rng(21)
    n, nb = 30000, 4
    tl = rng.integers(0, 60000, n).astype(np.uint32)
    sums = (rng.random((nb, n)) ** 3 * tl * 40).astype(np.uint64)
    sums[:, ::97] = 0
    sums[1, 5] = np.uint64(2 ** 45)                         # a mean above 1e6
    avg = [150, 101, 250, 33]
    names = [f"k141_{i} flag=1" if i % 3 else f"k141_{i}" for i in range(n)]
    bams = [f"/run/s{b}.bam" for b in range(nb)]
    for variance in (False, True):
        want = oracle.depth_tsv_ref(sums, avg, tl, names, bams, variance, False, 75, 1500)
        m, keep = _matrix(api, sums, avg, tl, names, 1500, nb)
        p = api.default_depth_params(min_contig_length=1500, threads=6)
        bn = (C.c_char_p * nb)(*[x.encode() for x in bams])
        buf, ln = C.c_void_p(), C.c_int64()
        assert L.rbg_depth_tsv(C.byref(m), bn, nb, C.byref(p), int(variance), C.byref(buf),
                               C.byref(ln)) == 0
        got = C.string_at(buf, ln.value)
        L.rbg_free_tsv(buf)
        assert got == want, variance
