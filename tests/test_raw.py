"""Raw DEFLATE (gzippy::decompress_raw, src/lib.rs:250): one RFC 1951 stream
with no gzip framing, decoded up to its final block; bytes after it are
ignored (decompress_raw_bytes, src/decompress/mod.rs:920).  Byte-exact, no
tolerance: the oracle and zlib (wbits -15) on the CPU, the device path
through gzgpu_inflate_raw against both on the GPU."""
import zlib

import numpy as np
import pytest

from gzippy_b200 import workloads as W
from oracle import pyoracle as O


def raw(plain: bytes, level: int, strategy: int = zlib.Z_DEFAULT_STRATEGY) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, -15, 8, strategy)
    return c.compress(plain) + c.flush()


def zraw(comp: bytes) -> bytes:
    d = zlib.decompressobj(-15)
    return d.decompress(comp)


def _cases(big: bool):
    out = []
    size = (24 << 20) if big else (256 << 10)
    for kind in (W.MARKOV, W.RANDOM, W.RUNS, W.RAMPS):
        p = W.content(kind, 700 + kind, size).tobytes()
        out.append((f"k{kind}-l6", p, raw(p, 6)))
    p = W.content(W.MARKOV, 711, size).tobytes()
    out.append(("fixed-l1", p, raw(p, 1, zlib.Z_FIXED)))
    out.append(("l9", p, raw(p, 9)))
    out.append(("empty", b"", raw(b"", 6)))
    out.append(("trailing", p[:4096], raw(p[:4096], 6) + b"\x00garbage after the final block"))
    return out


@pytest.mark.parametrize("name,plain,comp", _cases(False), ids=lambda x: x if isinstance(x, str) else "")
def test_oracle_raw_matches_zlib(name, plain, comp):
    st, got, _ = O.inflate_raw(comp, cap=len(plain) + 64)
    assert st == 0 and got == plain == zraw(comp)


def test_oracle_raw_rejects_cut_off_stream():
    p = W.content(W.MARKOV, 720, 64 << 10).tobytes()
    c = raw(p, 6)
    st, got, _ = O.inflate_raw(c[: len(c) // 2], cap=len(p) + 64)
    assert st != 0 and got is None


@pytest.mark.gpu
@pytest.mark.parametrize("big", [False, True])
def test_device_raw_matches_oracle_and_zlib(big):
    import gzippy_b200 as G
    cx = G.Context()
    try:
        for name, plain, comp in _cases(big):
            got = cx.inflate_raw(comp)
            assert got == plain == zraw(comp), name
            if not big:
                st, ref, _ = O.inflate_raw(comp, cap=len(plain) + 64)
                assert st == 0 and got == ref, name
        assert G.decompress_raw(_cases(False)[0][2]) == _cases(False)[0][1]
    finally:
        cx.close()


@pytest.mark.gpu
def test_device_raw_errors():
    import gzippy_b200 as G
    p = W.content(W.MARKOV, 721, 4 << 20).tobytes()
    c = raw(p, 6)
    cx = G.Context()
    try:
        with pytest.raises(G.GzippyError):
            cx.inflate_raw(b"")
        with pytest.raises(G.GzippyError):
            cx.inflate_raw(c[: len(c) // 2])          # cut off: no final block
        with pytest.raises(G.GzippyError):
            cx.inflate_raw(b"\x07" + c[1:])             # BTYPE 3 (reserved) in the first header
        # a gzip member is not raw DEFLATE: its header bytes are decoded as
        # DEFLATE and fail, as in the reference
        with pytest.raises(G.GzippyError):
            cx.inflate_raw(W.gzip_member(np.frombuffer(p[:65536], np.uint8), 6).tobytes())
        assert cx.inflate_raw(c) == p                    # the context still works
    finally:
        cx.close()


@pytest.mark.gpu
def test_device_zlib_matches_zlib():
    """decompress_zlib_turbo (src/decompress/mod.rs:895-914): the DEFLATE data
    between the 2-byte header and the Adler-32, neither checked."""
    import gzippy_b200 as G
    cx = G.Context()
    try:
        for kind, level, size in ((W.MARKOV, 6, 24 << 20), (W.RUNS, 9, 1 << 20), (W.RANDOM, 1, 64 << 10)):
            p = W.content(kind, 730 + kind, size).tobytes()
            z = zlib.compress(p, level)
            assert cx.inflate_zlib(z) == p == zlib.decompress(z)
        with pytest.raises(G.GzippyError):
            cx.inflate_zlib(b"\x78\x9c\x03")                  # under 6 bytes
    finally:
        cx.close()


def _stored_cases():
    p = W.content(W.MARKOV, 740, 3 << 20).tobytes()
    c = zlib.compressobj(6, zlib.DEFLATED, 31)
    flushed = b"".join(c.compress(p[i:i + 1000]) + c.flush(zlib.Z_SYNC_FLUSH)
                       for i in range(0, 200000, 1000)) + c.compress(p[200000:]) + c.flush()
    mixed = b"".join(W.content(k % 4, 741 + k, 1 << 20).tobytes() for k in range(24))
    return [("level0-mixed", mixed, W.gzip_member(np.frombuffer(mixed, np.uint8), 0).tobytes()),
            ("empty-stored-blocks", p, flushed)]


@pytest.mark.gpu
def test_device_stored_members():
    """Stored-only members (level 0, the stored-dominated case of
    parallel/stored_split.rs) and members with hundreds of empty stored
    blocks (sync flushes) decode byte-exact."""
    import gzippy_b200 as G
    cx = G.Context()
    try:
        for name, plain, comp in _stored_cases():
            assert cx.decompress(comp) == plain == zlib.decompress(comp, 31), name
    finally:
        cx.close()
