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
