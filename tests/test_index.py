"""Seek index (build_index + serialize_index, src/decompress/index.rs:55-141;
checkpoint rule of scan_deflate, src/decompress/scan_inflate.rs:46-130).

The oracle lists a member's blocks by decoding one block at a time and
applies the rule; it is pinned by resuming: decoding from every point's bit
with its window reproduces the output from that point's offset.  The device
builds the index from its parallel decode (each chunk logs the blocks it
decodes); its bytes must equal the oracle's exactly (integer work, no
tolerance), across chunk boundaries, speculative and sync starts."""
import zlib

import numpy as np
import pytest

from gzippy_b200 import workloads as W
from oracle import pyoracle as O


def member(kind: int, seed: int, size: int, level: int):
    p = W.content(kind, seed, size)
    return p.tobytes(), W.gzip_member(p, level).tobytes()


def mixed(seed: int, segs: int, seg: int, level: int):
    p = np.concatenate([W.content(k % 4, seed + k, seg) for k in range(segs)])
    return p.tobytes(), W.gzip_member(p, level).tobytes()


@pytest.mark.parametrize("kind,level,interval", [(W.MARKOV, 6, 256 << 10), (W.RUNS, 9, 0),
                                                 (W.MARKOV, 1, 100 << 10), (W.RAMPS, 6, 1 << 20)])
def test_oracle_index_points_resume(kind, level, interval):
    import gzippy_b200 as G
    plain, comp = member(kind, 900 + kind, 2 << 20, level)
    ix = O.seek_index(comp, plain, interval)
    doff, total, pts = G.parse_index(ix)
    _, hl = O.gzip_header_len(comp)
    assert doff == hl and total == len(plain) and len(pts) >= 1 and pts[0][1] > 0
    for b, o, win in pts:
        assert win == plain[o - 32768:o]
        st, res, ent = O.inflate_chunk(comp, hl * 8 + b, window=win, cap=len(plain) - o + 64)
        assert st == 0 and res.final_block and ent.astype(np.uint8).tobytes() == plain[o:]
    offs = [o for _, o, _ in pts]
    assert offs == sorted(set(offs)) and all(b - a >= interval for a, b in zip(offs, offs[1:]))


def test_oracle_index_without_points():
    import gzippy_b200 as G
    plain, comp = member(W.MARKOV, 930, 20 << 10, 6)       # shorter than one window
    doff, total, pts = G.parse_index(O.seek_index(comp, plain, 1 << 20))
    assert total == len(plain) and pts == [(0, 0, bytes(32768))]


CASES = [("markov-l6", lambda: member(W.MARKOV, 940, 16 << 20, 6), 1 << 20),
         ("mixed-l6", lambda: mixed(950, 8, 2 << 20, 6), 256 << 10),
         ("markov-l1-fixed", lambda: member(W.MARKOV, 960, 12 << 20, 1), 512 << 10),
         ("runs-l9-every-block", lambda: member(W.RUNS, 970, 6 << 20, 9), 0),
         ("short", lambda: member(W.MARKOV, 980, 20 << 10, 6), 1 << 20)]


@pytest.mark.gpu
@pytest.mark.parametrize("name,make,interval", CASES, ids=[c[0] for c in CASES])
def test_device_index_equals_oracle(name, make, interval):
    import gzippy_b200 as G
    plain, comp = make()
    cx = G.Context()
    try:
        got = cx.build_index(comp, interval)
    finally:
        cx.close()
    assert got == O.seek_index(comp, plain, interval), name


@pytest.mark.gpu
def test_device_index_rejects_what_the_reference_rejects():
    import gzippy_b200 as G
    from test_multiblock import multiblock
    plain, comp = member(W.MARKOV, 990, 1 << 20, 6)
    cx = G.Context()
    try:
        for bad in (comp + comp,                            # two members
                    multiblock("gz4", 2 << 20, 1 << 20, 991)[1],   # gzippy multi-block format
                    b"not gzip at all, not gzip at all",
                    zlib.compress(plain)):                  # zlib framing
            with pytest.raises(G.GzippyError):
                cx.build_index(bad, 1 << 20)
        assert cx.build_index(comp, 1 << 20) == O.seek_index(comp, plain, 1 << 20)
    finally:
        cx.close()
