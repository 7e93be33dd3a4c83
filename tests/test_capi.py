"""C ABI tests that need no GPU: the library loads, exports every declared
entry point, keeps the reference defaults, and its host-side ProbMinHash
stream tables reproduce the reference sketch through the register minimum the
kernel computes."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from rabbitbin_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_library_exports_every_declared_symbol():
    L = api.lib()
    declared = api.exported_symbols()
    assert "rbg_bin_graph" in declared and "rbg_build_pmh_winners" in declared
    for name in declared:
        assert hasattr(L, name), name
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        for name in set(re.findall(r"\b(rbg_[a-z0-9_]+)\s*\(", text)):
            assert hasattr(L, name), f"{hdr}: {name}"


def test_default_params_are_reference_defaults():
    p = api.default_params()
    assert (p.k, p.m, p.pmh_seed, p.gc_norm, p.win_bits) == (4, 500, 42, 1, 16)
    assert p.gc_norm_cap == 20.0 and p.max_edges == 200 and p.mutual == 1 and p.base_on == 1
    assert p.coverage == 0.95 and p.min_edge == 0.70 and p.w_comp == -1.0
    assert p.min_cv == 1.0 and p.neg_thr == -0.3 and p.depth_sim == 2 and p.depth_fuse == 1
    assert p.wjac_norm == 1 and p.fp_contract == 1 and p.abdfirst == 1


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_create_without_device_fails_cleanly():
    with pytest.raises(api.RbgError):
        api.Context(0)


def test_null_arguments_rejected():
    L = api.lib()
    assert L.rbg_default_params(None) == -1
    assert L.rbg_create(0, None) == -1
    assert L.rbg_free_graph(None) == -1
    ne = C.c_int32()
    assert L.rbg_pmh_stream_tables(5, 500, 42, 1, C.byref(ne), None, None, None) == -1
    assert L.rbg_pmh_stream_tables(4, 1, 42, 1, C.byref(ne), None, None, None) == -1


@pytest.mark.parametrize("m", [2, 3, 64, 500, 1000])
def test_stream_tables_reproduce_sketch(orc, m):
    """reg[r] = min_e (1/w_e) U_e(r), first-inserted on ties, and its winner,
    equal the sequential ProbMinHash4 state (registers and winners)."""
    codes, U, W = api.stream_tables(4, m)
    assert len(codes) == 136 and U.shape == (136, m)
    rng = np.random.default_rng(m)
    for _ in range(25):
        sel = np.sort(rng.choice(136, size=int(rng.integers(1, 137)), replace=False))
        w = rng.uniform(5e-6, 20.0, size=len(sel))
        regs, win = orc.pmh_elements(codes[sel].astype(np.uint64), w, m=m)
        hv = (1.0 / w)[:, None] * U[sel]
        best = np.argmin(hv, axis=0)
        assert np.array_equal(hv[best, np.arange(m)], regs)
        assert np.array_equal(W[sel[best], np.arange(m)], (win ^ (win >> 32)).astype(np.uint32))


def test_stream_tables_equal_weights_ties(orc):
    """Equal weights make offers comparable across elements; ties keep the
    first-inserted element exactly as the tracker's strict < does."""
    codes, U, W = api.stream_tables(4, 128)
    sel = np.arange(136)
    w = np.full(136, 0.5)
    regs, win = orc.pmh_elements(codes[sel].astype(np.uint64), w, m=128)
    hv = (1.0 / w)[:, None] * U[sel]
    best = np.argmin(hv, axis=0)
    assert np.array_equal(W[best, np.arange(128)], (win ^ (win >> 32)).astype(np.uint32))


def test_stream_tables_strict_mode_differs_only_in_rounding():
    _, U1, W1 = api.stream_tables(4, 500, fp_contract=1)
    _, U0, W0 = api.stream_tables(4, 500, fp_contract=0)
    assert np.array_equal(W1, W0)        # the RNG path never depends on rounding here
    rel = np.abs(U1 - U0) / np.maximum(U1, 1e-300)
    assert rel.max() < 1e-15
