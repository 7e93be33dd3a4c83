"""The library's DEFLATE decoder (rabbitbin_b200/csrc/inflate.cuh, run by the
device's BGZF kernel) compiled for the host and checked against zlib: every
block type (stored, fixed and dynamic Huffman), every zlib level and strategy,
empty and one-byte streams, BAM payloads, and damaged streams (which must end
with a status, checked here under AddressSanitizer)."""
import ctypes as C
import os
import subprocess
import zlib

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _build(tmp, asan):
    out = str(tmp / ("libinflate_asan.so" if asan else "libinflate.so"))
    flags = ["-fsanitize=address", "-fno-omit-frame-pointer", "-O1"] if asan else ["-O2"]
    subprocess.run(["g++", "-std=c++17", "-fPIC", "-shared"] + flags +
                   [os.path.join(HERE, "native", "inflate_host.cpp"), "-o", out], check=True)
    return out


@pytest.fixture(scope="module")
def dec(tmp_path_factory):
    lib = C.CDLL(_build(tmp_path_factory.mktemp("inflate"), False))
    lib.host_inflate.argtypes = [C.c_char_p, C.c_uint32, C.c_void_p, C.c_uint32]
    lib.host_crc32.argtypes = [C.c_char_p, C.c_uint32]
    lib.host_crc32.restype = C.c_uint32
    return lib


def _deflate(data, level=6, strategy=zlib.Z_DEFAULT_STRATEGY, wbits=-15, mem=8):
    c = zlib.compressobj(level, zlib.DEFLATED, wbits, mem, strategy)
    return c.compress(data) + c.flush()


def _run(dec, comp, n):
    out = (C.c_uint8 * max(n, 1))()
    rc = dec.host_inflate(comp, len(comp), out, n)
    return rc, bytes(out)[:n]


def _payloads():
    rng = np.random.default_rng(3)
    from rabbitbin_b200.synth import make_bam, bam_records
    bam = make_bam(np.array([4000, 9000], np.uint32), np.array([30.0, 10.0]), seed=4)
    raw = bam_records(bam)[0]
    text = b"".join(b"line %d of some text with repeats repeats repeats\n" % i for i in range(3000))
    return {
        "empty": b"",
        "one": b"A",
        "zeros": bytes(65280),
        "random": rng.integers(0, 256, 65280, dtype=np.uint8).tobytes(),
        "dna": bytes(rng.choice(list(b"ACGT"), 65000).astype(np.uint8)),
        "text": text[:65280],
        "bam": raw[:65280],
        "bam_tail": raw[-30000:],
        "runs": bytes(np.repeat(rng.integers(0, 4, 4000, dtype=np.uint8), 16)),
    }


def test_matches_zlib_all_levels_and_strategies(dec):
    strategies = [zlib.Z_DEFAULT_STRATEGY, zlib.Z_FILTERED, zlib.Z_HUFFMAN_ONLY, zlib.Z_RLE,
                  zlib.Z_FIXED]
    for name, data in _payloads().items():
        for level in range(10):
            for st in strategies:
                comp = _deflate(data, level, st)
                rc, out = _run(dec, comp, len(data))
                assert rc == 0 and out == data, (name, level, st, rc)


def test_small_windows_and_memlevels(dec):
    data = _payloads()["bam"]
    for wbits in (-9, -12, -15):
        for mem in (1, 5, 9):
            rc, out = _run(dec, _deflate(data, 6, zlib.Z_DEFAULT_STRATEGY, wbits, mem), len(data))
            assert rc == 0 and out == data


def test_flushed_multi_block_streams(dec):
    """Streams of many deflate blocks (sync / full flushes, a stored block in
    the middle), as some writers produce."""
    p = _payloads()
    c = zlib.compressobj(6, zlib.DEFLATED, -15)
    parts = [p["text"][:20000], p["random"][:3000], p["bam"][:30000], b"", p["zeros"][:5000]]
    comp = b""
    for i, part in enumerate(parts):
        comp += c.compress(part)
        comp += c.flush(zlib.Z_SYNC_FLUSH if i % 2 == 0 else zlib.Z_FULL_FLUSH)
    comp += c.flush()
    data = b"".join(parts)
    rc, out = _run(dec, comp, len(data))
    assert rc == 0 and out == data


def test_wrong_sizes_are_reported(dec):
    data = _payloads()["text"]
    comp = _deflate(data)
    assert _run(dec, comp, len(data) - 1)[0] == 7      # more output than ISIZE
    assert _run(dec, comp, len(data) + 1)[0] == 8      # less output than ISIZE
    assert _run(dec, comp[:len(comp) // 2], len(data))[0] == 1


def test_crc32(dec):
    """Segmented CRC (32 segments joined over GF(2)) against zlib's."""
    for data in _payloads().values():
        assert dec.host_crc32(data, len(data)) == zlib.crc32(data)
    rng = np.random.default_rng(2)
    for n in list(range(0, 80)) + [4095, 4096, 4097, 65535, 65536]:
        data = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert dec.host_crc32(data, n) == zlib.crc32(data), n


def test_damaged_streams_end_with_a_status(tmp_path):
    """Bit flips and truncations in every kind of stream: the decoder must
    return (any status) without reading or writing out of bounds (run under
    AddressSanitizer in a separate process)."""
    exe = str(tmp_path / "inflate_fuzz")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address",
                    "-fno-omit-frame-pointer", os.path.join(HERE, "native", "inflate_fuzz.cpp"),
                    "-o", exe], check=True)
    rng = np.random.default_rng(11)
    recs = []
    for name, data in _payloads().items():
        for level, st in ((1, zlib.Z_DEFAULT_STRATEGY), (9, zlib.Z_DEFAULT_STRATEGY),
                          (6, zlib.Z_FIXED), (0, zlib.Z_DEFAULT_STRATEGY)):
            comp = bytearray(_deflate(data, level, st))
            recs.append((bytes(comp), len(data)))
            for _ in range(12):
                bad = bytearray(comp)
                for _ in range(int(rng.integers(1, 4))):
                    if len(bad):
                        i = int(rng.integers(0, len(bad)))
                        bad[i] ^= 1 << int(rng.integers(0, 8))
                recs.append((bytes(bad), len(data)))
                recs.append((bytes(bad[:int(rng.integers(0, len(bad) + 1))]), len(data)))
                recs.append((bytes(bad), int(rng.integers(0, 65537))))
    path = tmp_path / "streams.bin"
    with open(path, "wb") as f:
        for blob, n in recs:
            f.write(len(blob).to_bytes(4, "little") + n.to_bytes(4, "little") + blob)
    r = subprocess.run([exe, str(path)], capture_output=True, text=True,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=0"))
    assert r.returncode == 0, r.stderr[-3000:]
    runs, ok = map(int, r.stdout.split())
    assert runs == len(recs) and ok >= len(_payloads()) * 4
