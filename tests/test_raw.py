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


def _zeros_deflate(n: int, wbits: int) -> bytes:
    c = zlib.compressobj(6, zlib.DEFLATED, wbits)
    z = bytes(16 << 20)
    return b"".join(c.compress(z) for _ in range(n // len(z))) + c.flush()


@pytest.mark.gpu
def test_device_raw_and_zlib_high_ratio_grow_the_page_pool():
    """256 MiB of zeros (about 1000:1) as raw DEFLATE and as zlib.  These
    formats carry no ISIZE, so the page pool starts at 4x the input, far too
    small: the chunks that run out of pages are decoded again in a grown pool
    (up to deflate's 1032:1 ceiling), and the output is exact."""
    import ctypes
    import gzippy_b200 as G
    n = 256 << 20
    for wbits, entry in ((-15, "gzgpu_inflate_raw"), (15, "gzgpu_inflate_zlib")):
        comp = np.frombuffer(_zeros_deflate(n, wbits), np.uint8)
        assert comp.size * 500 < n
        cx = G.Context()          # a fresh pool, sized from the input alone
        try:
            out = np.full(n + 64, 0xA5, np.uint8)
            got = ctypes.c_size_t(0)
            rc = getattr(cx._lib, entry)(cx._h, comp.ctypes.data, comp.size, out.ctypes.data,
                                         out.size, ctypes.byref(got))
            assert rc == G.OK and got.value == n, (entry, rc)
            assert not out[:n].any() and out[n] == 0xA5
            assert cx.stats().pool_regrows >= 1
        finally:
            cx.close()


@pytest.mark.gpu
def test_device_member_over_4gib_with_wrapped_isize():
    """A gzip member of 4 GiB + 1 MiB: its ISIZE trailer holds the size mod
    2^32 (1 MiB), which sizes the page pool far too small.  The decode grows
    the pool, the trailer check compares sizes mod 2^32 as RFC 1952 defines
    ISIZE, and every byte lands in place (a period-1024 pattern, checked on
    the device)."""
    import torch
    import gzippy_b200 as G
    n = (4 << 30) + (1 << 20)
    rng = np.random.default_rng(5)
    blk = rng.integers(0, 256, 1024, dtype=np.uint8)
    piece = np.tile(blk, 65536).tobytes()            # 64 MiB, a whole number of periods
    c = zlib.compressobj(1, zlib.DEFLATED, 31)
    parts = [c.compress(piece) for _ in range(n // len(piece))]
    parts.append(c.compress(piece[: n % len(piece)]))
    parts.append(c.flush())
    comp = np.frombuffer(b"".join(parts), np.uint8)
    assert int.from_bytes(comp[-4:].tobytes(), "little") == n % (1 << 32)
    cx = G.Context()
    try:
        d_in = torch.zeros(comp.size + 1024, dtype=torch.uint8, device="cuda")
        d_in[: comp.size] = torch.from_numpy(comp).cuda()
        d_out = torch.empty(n + 4096, dtype=torch.uint8, device="cuda")
        got = cx.decompress_device(d_in.data_ptr(), comp.size, d_out.data_ptr(), d_out.numel())
        assert got == n
        assert cx.stats().pool_regrows >= 1
        want = torch.from_numpy(blk).cuda().repeat(n // 1024 + 1)[:n]
        assert torch.equal(d_out[:n], want)
        del want, d_out, d_in
        torch.cuda.empty_cache()
    finally:
        cx.close()
