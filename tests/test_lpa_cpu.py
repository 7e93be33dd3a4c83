"""Label propagation on the CPU: the correctly rounded exp / log of the device
sweep (ddmath.cuh, host build), the restatement oracle/lpa.py against the
reference's own cluster_by_propagation (oracle/_ref) and both against the
committed golden labels (tests/golden/lpa.npz, made by make_golden.py --lpa)."""
import math
import os
import subprocess
import sys
from decimal import Decimal, getcontext

import numpy as np
import pytest

from oracle import lpa

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
DDMATH = os.path.join(ROOT, "rabbitbin_b200", "csrc", "ddmath.cuh")

_DRIVER = r'''
#include "ddmath.cuh"
#include <cstdio>
#include <cstdlib>
int main(int argc, char **argv) {
  // argv[1]: "exp" or "log"; doubles (hex) on stdin, results (hex) on stdout
  const bool is_exp = argv[1][0] == 'e';
  char buf[64];
  while (scanf("%63s", buf) == 1) {
    const double x = strtod(buf, nullptr);
    const double y = is_exp ? rbg::dd::exp_cr(x) : rbg::dd::log_cr(x);
    printf("%a\n", y);
  }
}
'''


@pytest.fixture(scope="module")
def ddmath_bin(tmp_path_factory):
    d = tmp_path_factory.mktemp("ddmath")
    src = d / "drv.cpp"
    src.write_text(_DRIVER)
    exe = d / "drv"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-mfma",
                    "-I", os.path.dirname(DDMATH), str(src), "-o", str(exe)], check=True)
    return str(exe)


def _run(exe, kind, xs):
    inp = "\n".join(float(x).hex() for x in xs) + "\n"
    r = subprocess.run([exe, kind], input=inp, capture_output=True, text=True, check=True)
    return [float.fromhex(t) for t in r.stdout.split()]


def _cr(dv):
    return float(dv)            # Decimal -> float rounds to nearest even, subnormals included


def test_exp_correctly_rounded(ddmath_bin):
    getcontext().prec = 80
    rng = np.random.default_rng(11)
    xs = list(-rng.uniform(0, 745.5, 2500)) + list(-rng.uniform(0, 1e-3, 300)) + [
        0.0, -0.0, -1e-300, -5e-324, -0.5, -1.0, -math.log(2), -708.39, -708.4, -709.0, -709.5,
        -720.0, -744.0, -744.44, -745.0, -745.1332, -745.1333, -745.2, -746.0, 1.0, 0.5, 700.0]
    got = _run(ddmath_bin, "exp", xs)
    bad = [(x, g) for x, g in zip(xs, got) if g != _cr(Decimal(x).exp())]
    assert not bad, bad[:5]
    # agreement with the C library's exp, which the reference calls
    agree = np.mean([g == math.exp(x) for x, g in zip(xs, got)])
    assert agree > 0.995


def test_log_correctly_rounded(ddmath_bin):
    getcontext().prec = 80
    rng = np.random.default_rng(12)
    w = rng.uniform(0, 1, 3000).astype(np.float32)
    w = w[(w > 0) & (w <= np.float32(1) - np.float32(1e-6))]
    xs = [1.0 - float(v) for v in w] + [1.0, 1e-6, 0.5, 0.25, 1 - 2 ** -24, 2 ** -20, 0.3]
    got = _run(ddmath_bin, "log", xs)
    bad = [(x, g) for x, g in zip(xs, got) if g != _cr(Decimal(x).ln())]
    assert not bad, bad[:5]
    # the per-arc quantity is stored as float: equal to the C library's in every case here
    assert all(np.float32(g) == np.float32(math.log(x)) for x, g in zip(xs, got))


def _graph(n, seed, k=16, groups=8):
    rng = np.random.default_rng(seed)
    g = rng.integers(0, groups, n)
    src, dst, w = [], [], []
    for i in range(n):
        for j in rng.choice(n, k, replace=False):
            if j > i and (g[i] == g[j] or rng.random() < 0.15):
                src.append(i)
                dst.append(j)
                w.append(rng.uniform(0.7, 1.0) if g[i] == g[j] else rng.uniform(0, 0.9))
    w = np.array(w, np.float32)
    w[::37] = 0.0                 # dropped from the incidence lists
    w[::53] = 1.0                 # clamped to 1 - 1e-6
    return np.array(src, np.uint32), np.array(dst, np.uint32), w


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("sync", [False, True])
def test_restatement_matches_reference(ref_lib, seed, sync, monkeypatch):
    n = 240
    s, d, w = _graph(n, seed)
    order = ref_lib.lpa_node_order(n, seed + 1)
    if sync:
        monkeypatch.setenv("RABBIT_PAR_LPA", "1")
    a = ref_lib.label_propagation(n, s, d, w, seed=seed + 1)
    b = lpa.label_propagation(n, s, d, w, order, synchronous=sync)
    assert (a == b).all()


_RULES_CHILD = r'''
import sys, numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import oracle
from oracle import lpa
from test_lpa_cpu import _graph
rule = sys.argv[2]
n = 200
s, d, w = _graph(n, 5)
a = oracle.ref().label_propagation(n, s, d, w, seed=3)
b = lpa.label_propagation(n, s, d, w, oracle.ref().lpa_node_order(n, 3), rule=lpa.RULES[rule])
sys.exit(0 if (a == b).all() else 1)
'''


@pytest.mark.parametrize("rule", ["tail", "logsum", "sum", "mean", "max"])
def test_score_rules_match_reference(ref_lib, rule):
    # the reference reads RABBIT_LPA_SCORE when its library loads: a fresh process per rule
    env = dict(os.environ, RABBIT_LPA_SCORE=rule)
    env.pop("RABBIT_PAR_LPA", None)
    r = subprocess.run([sys.executable, "-c", _RULES_CHILD, ROOT, rule], env=env,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("name", ["small_path_s5", "fused_s3_m96"])
def test_restatement_matches_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    L = np.load(os.path.join(GOLDEN, "lpa.npz"))
    n = len(g["offsets"]) - 1
    order = L[f"{name}_order_1"]
    got = lpa.label_propagation(n, g["src"], g["dst"], g["score"], order)
    assert (got == L[f"{name}_gs_1"]).all()


def test_reference_harness_matches_golden(ref_lib, monkeypatch):
    monkeypatch.delenv("RABBIT_PAR_LPA", raising=False)
    L = np.load(os.path.join(GOLDEN, "lpa.npz"))
    for name in ["small_path_s5", "fused_s20_m64"]:
        g = np.load(os.path.join(GOLDEN, name + ".npz"))
        n = len(g["offsets"]) - 1
        assert (ref_lib.lpa_node_order(n, 1) == L[f"{name}_order_1"]).all()
        got = ref_lib.label_propagation(n, g["src"], g["dst"], g["score"], seed=7)
        assert (got == L[f"{name}_gs_7"]).all()


def test_negative_score_is_an_error(ref_lib):
    with pytest.raises(ValueError):
        ref_lib.label_propagation(3, [0], [1], np.array([-0.5], np.float32))
