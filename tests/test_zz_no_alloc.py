"""The no-allocation entry point (gzgpu_decompress_device_noalloc).

Some callers cannot call cudaMalloc: code under a pool-only allocator that
must not grow, real-time paths that cannot take the device-wide
synchronisation cudaMalloc/cudaFree may cause, or processes whose device
memory is reserved up front by another framework.  For them the library decodes with a fixed
device array instead of allocating.  This test calls that entry point
through the C ABI and checks its output byte for byte against the regular
entry point (gzgpu_decompress) and against the plaintext the stream was
made from -- integer work, so equality is exact -- on two calls in a row,
since every call reuses the same array.  It lives in its own file, collected
last, and passes in a fresh process as well as after the other tests."""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gz(data: bytes, level: int = 6, strategy: int = zlib.Z_DEFAULT_STRATEGY) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, 31, 8, strategy)
    return c.compress(data) + c.flush()


def _cases():
    from gzippy_b200 import workloads as W
    text = W.content(W.MARKOV, 21, 1 << 20).tobytes()
    rnd = W.content(W.RANDOM, 22, 600_000).tobytes()
    runs = W.content(W.RUNS, 23, 2 << 20).tobytes()
    ramps = W.content(W.RAMPS, 24, 300_000).tobytes()
    # name -> (gzip stream, the plaintext it decodes to)
    return {
        "text_l6": (_gz(text, 6), text),
        "random_stored": (_gz(rnd, 6), rnd),
        "runs_l9": (_gz(runs, 9), runs),
        "text_fixed_l1": (_gz(text[:500_000], 1, zlib.Z_FIXED), text[:500_000]),
        "multi_member": (_gz(ramps, 6) + _gz(b"") + _gz(text[:100_000], 9),
                         ramps + text[:100_000]),
        "trailing_garbage": (_gz(ramps[:50_000], 6) + b"\x00not a member", ramps[:50_000]),
        "empty_member": (_gz(b""), b""),
    }


def _device(blob: bytes, out_cap: int):
    import torch
    d_in = torch.zeros(len(blob) + 1024, dtype=torch.uint8, device="cuda")
    if blob:
        d_in[: len(blob)] = torch.frombuffer(bytearray(blob), dtype=torch.uint8).cuda()
    d_out = torch.empty(max(out_cap, 1), dtype=torch.uint8, device="cuda")
    return d_in, d_out


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    import gzippy_b200 as G
    ctx = G.Context()
    for name, (blob, plain) in _cases().items():
        ref = ctx.decompress(blob)
        assert ref == plain, name
        d_in, d_out = _device(blob, len(ref) + 64)
        for call in range(2):
            d_out.fill_(0xA5)  # stale bytes cannot pass for output
            torch.cuda.synchronize()
            n = G.decompress_device_noalloc(d_in.data_ptr(), len(blob), d_out.data_ptr(),
                                            d_out.numel())
            assert n == len(ref), (name, call)
            got = d_out[:n].cpu().numpy().tobytes()
            assert got == ref and got == plain, (name, call)
    ctx.close()


def test_noalloc_out_too_small_reports_the_whole_stream():
    """A multi-member stream whose second member does not fit: the call
    reports the exact size of all members, and writes nothing past out_cap."""
    import gzippy_b200 as G
    from gzippy_b200 import workloads as W
    parts = [W.content(t, 30 + t, 150_000 + 10_000 * t).tobytes() for t in range(4)]
    blob = b"".join(_gz(p, 6) for p in parts)
    total = sum(len(p) for p in parts)
    d_in, d_out = _device(blob, total + 64)
    for cap in (len(parts[0]) + 10, 1000, total - 1):
        for _ in range(2):
            d_out.fill_(0xA5)
            with pytest.raises(G.GzippyError) as ei:
                G.decompress_device_noalloc(d_in.data_ptr(), len(blob), d_out.data_ptr(), cap)
            assert ei.value.code == G.OUT_TOO_SMALL
            assert ei.value.needed == total, cap
            assert bool(d_out[cap:].eq(0xA5).all())
    # with the size it reported, the same call succeeds
    n = G.decompress_device_noalloc(d_in.data_ptr(), len(blob), d_out.data_ptr(), total)
    assert n == total and d_out[:n].cpu().numpy().tobytes() == b"".join(parts)


def _code(fn):
    import gzippy_b200 as G
    try:
        fn()
    except G.GzippyError as e:
        return e.code
    return 0


def test_noalloc_limits_and_errors():
    import gzippy_b200 as G
    from gzippy_b200 import workloads as W
    big = _gz(W.content(W.RANDOM, 25, G.NOALLOC_MAX_OUT + 100_000).tobytes(), 6)
    d_in, d_out = _device(big, G.NOALLOC_MAX_OUT + 200_000)
    with pytest.raises(G.GzippyError) as ei:
        G.decompress_device_noalloc(d_in.data_ptr(), len(big), d_out.data_ptr(), d_out.numel())
    assert ei.value.code == G.NOALLOC_TOO_LARGE
    good = _gz(W.content(W.MARKOV, 26, 200_000).tobytes(), 6)
    crc_bad = bytearray(good)
    crc_bad[-8] ^= 1
    size_bad = bytearray(good)
    size_bad[-3] ^= 1
    ctx = G.Context()
    # each corrupt input fails with the status the regular entry point gives
    for blob in (bytes(crc_bad), bytes(size_bad), good[:-40], good[: len(good) // 2]):
        d_in, d_out = _device(blob, 300_000)
        want = _code(lambda: ctx.decompress(blob))
        assert want != 0
        for _ in range(2):
            got = _code(lambda: G.decompress_device_noalloc(d_in.data_ptr(), len(blob),
                                                            d_out.data_ptr(), d_out.numel()))
            assert got == want
    ctx.close()
    # output buffer too small: reported, not overrun
    d_in, d_out = _device(good, 300_000)
    d_out.fill_(0xA5)
    with pytest.raises(G.GzippyError) as ei:
        G.decompress_device_noalloc(d_in.data_ptr(), len(good), d_out.data_ptr(), 1000)
    assert ei.value.code == G.OUT_TOO_SMALL
    assert bool(d_out[1000:].eq(0xA5).all())
    d_in, d_out = _device(b"plain text", 64)
    assert G.decompress_device_noalloc(d_in.data_ptr(), 10, d_out.data_ptr(), 64) == 0
    # a good call after the failures still decodes correctly
    d_in, d_out = _device(good, 300_000)
    n = G.decompress_device_noalloc(d_in.data_ptr(), len(good), d_out.data_ptr(), d_out.numel())
    assert d_out[:n].cpu().numpy().tobytes() == zlib.decompress(good, 31)
