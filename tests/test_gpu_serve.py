"""Serving form (rbg_server_*): requests submitted while others are on the GPU
are folded into shared launches, and each result is the same as the
single-assembly call on that assembly alone (edges and weights bit for bit)."""
import threading
import time

import numpy as np
import pytest

from rabbitbin_b200 import api
from rabbitbin_b200.synth import make_assembly

pytestmark = pytest.mark.gpu

KEYS = ("src", "dst", "scomp", "score")


@pytest.fixture(scope="module")
def requests_mix():
    """12 assemblies of mixed size, S and m (small and fused paths)."""
    rng = np.random.default_rng(44)
    out = []
    for i in range(12):
        n = int(rng.choice([400, 900, 1800, 3200]))
        S = int(rng.choice([3, 5, 10, 30]))
        m = int(rng.choice([250, 500, 1000]))
        a = make_assembly(max(5, n // 300), n, S, seed=900 + i, absent_frac=0.1)
        buf, offs = a.concat()
        kw = dict(m=m, force_path=2 if n > 2500 else 0)
        out.append((buf, offs, a.depth, kw))
    return out


def _alone(ctx, reqs):
    return [ctx.bin_graph(b, o, d, api.default_params(**kw)) for b, o, d, kw in reqs]


def _same(got, want, i):
    assert got["b0"] == want["b0"] and got["sim_cutoff"] == want["sim_cutoff"], i
    for k in KEYS:
        assert np.array_equal(got[k], want[k]), (i, k)


def _serve(srv, reqs, threads=4):
    """Submit from several threads with small random gaps; wait for all."""
    ids = [None] * len(reqs)
    params = [api.default_params(**kw) for _, _, _, kw in reqs]

    def client(t):
        rng = np.random.default_rng(t)
        for i in range(t, len(reqs), threads):
            time.sleep(float(rng.uniform(0.0, 0.02)))
            b, o, d, _ = reqs[i]
            ids[i] = srv.submit(b, o, d, params[i])

    th = [threading.Thread(target=client, args=(t,)) for t in range(threads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return [srv.wait(r, timeout=600.0) for r in ids]


def test_served_equals_alone(gpu_ctx, requests_mix):
    want = _alone(gpu_ctx, requests_mix)
    srv = api.Server(workers=2, max_batch=8)
    try:
        got = _serve(srv, requests_mix)
        # a second wave on the same workers (reused buffers and graphs)
        again = _serve(srv, requests_mix[::-1])[::-1]
    finally:
        srv.close()
    for i, ((g, st), w) in enumerate(zip(got, want)):
        _same(g, w, i)
        assert st["latency_ms"] >= st["service_ms"] >= 0.0
    for i, ((g, _), w) in enumerate(zip(again, want)):
        _same(g, w, i)
    assert max(st["batch_size"] for _, st in got + again) >= 2, "no request was folded"


def test_plain_mode_equals_alone(gpu_ctx, requests_mix):
    reqs = requests_mix[:5]
    want = _alone(gpu_ctx, reqs)
    srv = api.Server(plain=True)
    try:
        got = _serve(srv, reqs, threads=2)
    finally:
        srv.close()
    for i, ((g, st), w) in enumerate(zip(got, want)):
        _same(g, w, i)
        assert st["batch_size"] == 1


def test_server_rejections(requests_mix):
    b, o, d, kw = requests_mix[0]
    srv = api.Server(workers=1, hbm_budget=1 << 20)      # 1 MiB: nothing fits
    try:
        with pytest.raises(api.RbgError) as e:
            srv.submit(b, o, d, api.default_params(**kw))
        assert e.value.code == -2
    finally:
        srv.close()
    srv = api.Server(workers=1)
    try:
        with pytest.raises(api.RbgError) as e:
            srv.submit(b, o, d, api.default_params(m=1))
        assert e.value.code == -1
        with pytest.raises(api.RbgError):
            srv.wait(12345, timeout=0.0)                    # unknown id
        rid = srv.submit(b, o, d, api.default_params(**kw))
        g, st = srv.wait(rid)                               # still serves after rejections
        assert len(g["src"]) > 0 and st["batch_size"] == 1
    finally:
        srv.close()


def test_small_requests_overlap_a_large_batch(gpu_ctx):
    """Continuous admission: small requests submitted while a large one runs
    start on the small-request lane before the large one finishes, and every
    result equals rbg_bin_graph on that assembly alone."""
    from rabbitbin_b200.synth import make_assembly
    big = make_assembly(60, 30000, 5, seed=611)
    smalls = [make_assembly(8, 400 + 50 * k, 5, seed=620 + k) for k in range(4)]
    reqs = [(a,) + a.concat() for a in [big] + smalls]
    want = [gpu_ctx.bin_graph(b, o, a.depth) for a, b, o in reqs]
    srv = api.Server(workers=2, small_pairs=1_000_000)
    try:
        ids = [srv.submit(b, o, a.depth) for a, b, o in reqs]
        got = [srv.wait(i, timeout=600.0) for i in ids]
    finally:
        srv.close()
    for k, ((g, st), w) in enumerate(zip(got, want)):
        for key in ("src", "dst", "scomp", "score"):
            assert np.array_equal(g[key], w[key]), (k, key)
    big_st = got[0][1]
    assert big_st["worker"] == 0
    for g, st in got[1:]:
        assert st["worker"] == 1
        assert st["submit_s"] + st["queue_ms"] / 1000.0 < big_st["done_s"], \
            "a small request waited for the large batch"
