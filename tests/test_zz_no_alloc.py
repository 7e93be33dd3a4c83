"""The allocation-free sketch entry point against the regular one.

rbg_build_pmh_winners_noalloc exists for callers that cannot allocate device
memory: they hand in device buffers and the library works inside a static
array it reserved when it was loaded.  Its winner rows must equal those of
rbg_build_pmh_winners (bit-exact, the tolerance of every sketch test here),
on two calls in a row, alone in a fresh process or after the other tests.
This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly

pytestmark = pytest.mark.gpu


def _noalloc(buf, offs, m, **kw):
    import torch
    L = api.lib()
    n = len(offs) - 1
    nbytes = (len(buf) + 15) // 16 * 16
    seq = torch.zeros(max(nbytes, 16), dtype=torch.uint8, device="cuda")
    if len(buf):
        seq[:len(buf)] = torch.frombuffer(bytearray(buf), dtype=torch.uint8).cuda()
    off = torch.from_numpy(np.ascontiguousarray(offs, np.int64)).cuda()
    out = torch.zeros((n, m), dtype=torch.int32, device="cuda")
    p = api.default_params(m=m, **kw)
    err = C.create_string_buffer(256)
    rc = L.rbg_build_pmh_winners_noalloc(C.byref(p), seq.data_ptr(), off.data_ptr(), n,
                                         int(offs[-1]), out.data_ptr(), None, err, 256)
    assert rc == 0, err.value.decode()
    return out.cpu().numpy().view(np.uint32)


def _call_raw(offs_list, nbases, **kw):
    """Status and message of one call on caller-built offsets (no output check)."""
    import torch
    L = api.lib()
    n = len(offs_list) - 1
    seq = torch.full(((nbases + 15) // 16 * 16 + 16,), ord("A"), dtype=torch.uint8, device="cuda")
    off = torch.tensor(offs_list, dtype=torch.int64, device="cuda")
    out = torch.zeros(max(n * 500, 16), dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(256)
    rc = L.rbg_build_pmh_winners_noalloc(C.byref(api.default_params(**kw)), seq.data_ptr(),
                                         off.data_ptr(), n, nbases, out.data_ptr(), None,
                                         err, 256)
    torch.cuda.synchronize()
    return rc, err.value


@pytest.mark.parametrize("m,gc", [(500, 1), (96, 1), (500, 2), (2000, 0)])
def test_noalloc_matches_regular_entry_point(m, gc):
    ctx = api.Context(0)
    try:
        for seed in (1, 2):                     # two calls in a row
            asm = make_assembly(10, 400 if seed == 1 else 250, 0, seed=seed, n_frac=0.01)
            seqs = [b"", b"ACG", b"NNNN", b"ACGT" * 9] + asm.seqs
            offs = np.zeros(len(seqs) + 1, np.int64)
            offs[1:] = np.cumsum([len(s) for s in seqs])
            buf = b"".join(seqs)
            want = ctx.build_pmh_winners(buf, offs, api.default_params(m=m, gc_norm=gc))
            got = _noalloc(buf, offs, m, gc_norm=gc)
            assert np.array_equal(got, want), f"seed {seed}: winner rows differ"
    finally:
        ctx.close()


def test_noalloc_rejects_oversized_request():
    import torch
    L = api.lib()
    n = 1 << 20                                    # 1M contigs: far beyond the array
    seq = torch.zeros(16, dtype=torch.uint8, device="cuda")
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(256)
    rc = L.rbg_build_pmh_winners_noalloc(C.byref(api.default_params()), seq.data_ptr(),
                                         off.data_ptr(), n, 0, out.data_ptr(), None, err, 256)
    assert rc == -1 and b"scratch" in err.value


def test_noalloc_rejects_bad_offsets():
    """Offsets that decrease (though every value lies in [0, nbases]) or that
    leave [0, nbases] are refused by the device-side check before any sketch
    work; a well-formed call right after still succeeds."""
    rc, msg = _call_raw([0, 600, 300, 1000], 1000)
    assert rc == -1 and b"never decrease" in msg
    rc, msg = _call_raw([0, 400, 1000, 1000], 900)
    assert rc == -1
    rc, msg = _call_raw([0, 500, 1000], 1000)
    assert rc == 0, msg


def test_noalloc_rejects_oph_metric():
    rc, msg = _call_raw([0, 500, 1000], 1000, oph_k=8)
    assert rc == -1 and b"ProbMinHash" in msg
