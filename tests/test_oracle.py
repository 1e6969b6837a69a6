"""Oracle pins: the CPU restatement against the reference's GZBLK01
known-answer blocks and against system zlib on every content type/level."""
import glob
import os
import struct
import zlib

import numpy as np
import pytest

from oracle import pyoracle as O
from gzippy_b200 import workloads as W
from conftest import REFERENCE_BLOCKS


def _gzblk01(path):
    """GZBLK01 layout (tools/extract_blocks/src/main.rs:7-30 of the reference)."""
    b = open(path, "rb").read()
    (magic, idx, btype, bitoff, bitlen, bytelen, declen, predlen, nl, nd, mll, mdl, mc, crc,
     _res) = struct.unpack_from("<8sIIQQQIIHHBBHII", b, 0)
    assert magic == b"GZBLK01\0" and btype == 2
    o = 64
    pred = b[o:o + predlen]; o += predlen
    comp = b[o:o + bytelen]; o += bytelen
    dec = b[o:o + declen]; o += declen
    lcl = np.frombuffer(b[o:o + nl], np.uint8); o += nl
    dcl = np.frombuffer(b[o:o + nd], np.uint8)
    return dict(idx=idx, bitoff=bitoff, bitlen=bitlen, pred=pred, comp=comp, dec=dec,
                lcl=lcl, dcl=dcl, crc=crc)


BLOCKS = sorted(glob.glob(os.path.join(REFERENCE_BLOCKS, "*.bin")))


@pytest.mark.skipif(not BLOCKS, reason="reference corpus not mounted")
@pytest.mark.parametrize("path", BLOCKS, ids=[os.path.basename(p) for p in BLOCKS])
def test_gzblk01_known_answer(path):
    k = _gzblk01(path)
    st, r, out = O.inflate_chunk(k["comp"], k["bitoff"], k["bitoff"] + 1, window=k["pred"],
                                 cap=len(k["dec"]) + 1024)
    assert st == O.OK
    assert r.end_bit == k["bitoff"] + k["bitlen"]          # block length in bits
    assert r.n_blocks == 1 and r.marker_end == 0
    assert out.astype(np.uint8).tobytes() == k["dec"]
    assert O.crc32(k["dec"]) == k["crc"]
    st, lcl, dcl = O.dynamic_lengths(k["comp"], k["bitoff"])
    assert st == O.OK and (lcl == k["lcl"]).all() and (dcl == k["dcl"]).all()
    # the block finder accepts the true block start (test_block_finder_at_oracle_positions)
    assert O.is_dynamic_candidate(k["comp"], k["bitoff"])
    first, seek = O.find_blocks(k["comp"], max(0, k["bitoff"] - 4096), k["bitoff"] + 1)
    assert k["bitoff"] in set(first.tolist())


@pytest.mark.skipif(not BLOCKS, reason="reference corpus not mounted")
def test_gzblk01_markers_resolve_to_window():
    """Decoding window-absent emits markers that resolve against the
    predecessor window to the known answer (replace_markers.rs:7-23)."""
    for path in BLOCKS[:6]:
        k = _gzblk01(path)
        st, r, out = O.inflate_chunk(k["comp"], k["bitoff"], k["bitoff"] + 1, markers=True,
                                     cap=len(k["dec"]) + 1024)
        assert st == O.OK
        w = np.frombuffer(k["pred"], np.uint8)
        res = np.where(out < 256, out, w[(out.astype(np.int64) - 32768).clip(0, 32767)])
        assert res.astype(np.uint8).tobytes() == k["dec"]


def test_crc32_and_combine():
    rng = np.random.default_rng(0)
    for n in (0, 1, 7, 8, 9, 1000, 65537):
        a = rng.integers(0, 256, n, dtype=np.uint8)
        assert O.crc32(a) == zlib.crc32(a.tobytes())
    a = rng.integers(0, 256, 5000, dtype=np.uint8).tobytes()
    for cut in (0, 1, 100, 4999, 5000):
        c1, c2 = zlib.crc32(a[:cut]), zlib.crc32(a[cut:])
        assert O.crc32_combine(c1, c2, len(a) - cut) == zlib.crc32(a)
    # x^(8n) * x^(8m) == x^(8(n+m))
    lib = O.lib()
    assert lib.orc_gf2_mulmod(lib.orc_x_pow_8n(3), lib.orc_x_pow_8n(5)) == lib.orc_x_pow_8n(8)


@pytest.mark.parametrize("ctype", [W.MARKOV, W.RANDOM, W.RUNS, W.RAMPS])
@pytest.mark.parametrize("level", [1, 6, 9])
def test_oracle_matches_zlib(ctype, level):
    p = W.content(ctype, 11 + ctype, 1 << 20)
    c = W.gzip_member(p, level)
    assert zlib.decompress(c.tobytes(), 31) == p.tobytes()
    st, out = O.decompress(c)
    assert st == O.OK and out.tobytes() == p.tobytes()
    st, out, stats = O.decompress_chunked(c, chunk_bytes=32 << 10, threads=4)
    assert st == O.OK and out.tobytes() == p.tobytes()


def test_block_types_follow_level():
    """level 1 -> fixed-Huffman blocks, 6/9 -> dynamic, random -> stored."""
    p = W.content(W.MARKOV, 3, 1 << 20)
    for level, kind in ((1, "n_fixed"), (6, "n_dynamic"), (9, "n_dynamic")):
        c = W.gzip_member(p, level)
        _, hl = O.gzip_header_len(c)
        st, r, _ = O.inflate_chunk(c, hl * 8, cap=2 << 20)
        assert st == O.OK and r.final_block
        assert getattr(r, kind) >= r.n_blocks - 1
    c = W.gzip_member(W.content(W.RANDOM, 3, 1 << 20), 6)
    _, hl = O.gzip_header_len(c)
    st, r, _ = O.inflate_chunk(c, hl * 8, cap=2 << 20)
    assert r.n_stored >= r.n_blocks - 1


def test_finder_scan_equals_per_bit_predicate():
    """The skip-LUT scan returns exactly the bits the full predicate accepts
    (branchless_scan_matches_scalar, blockfinder_validation.rs:1237)."""
    c = W.gzip_member(W.content(W.MARKOV, 5, 256 << 10), 6)
    lo, hi = 8 * 20, 8 * 20 + 40000
    first, seek = O.find_blocks(c, lo, hi)
    dyn = [b for b in range(lo, hi) if O.is_dynamic_candidate(c, b)]
    got_dyn = [int(f) for f, s in zip(first, seek) if f == s and O.is_dynamic_candidate(c, int(f))]
    assert got_dyn == dyn


def test_finder_finds_true_boundaries():
    p = W.content(W.MARKOV, 9, 2 << 20)
    c = W.gzip_member(p, 6)
    _, hl = O.gzip_header_len(c)
    # walk the true block boundaries with the decoder
    bounds, pos = [], hl * 8
    while True:
        st, r, _ = O.inflate_chunk(c, pos, pos + 1, cap=4 << 20)
        assert st == O.OK
        bounds.append((pos, r.final_block))
        if r.final_block:
            break
        pos = r.end_bit
    first, seek = O.find_blocks(c, hl * 8, c.size * 8)
    found = set(first.tolist())
    dyn_bounds = [b for b, fin in bounds[1:] if not fin]
    assert all(b in found for b in dyn_bounds)


def test_member_scan_multi():
    parts = [W.gzip_member(W.content(t % 4, t, 100000), 6) for t in range(5)]
    data = np.concatenate(parts)
    ms = O.scan_members(data)
    assert [m.start for m in ms] == list(np.cumsum([0] + [p.size for p in parts[:-1]]))
    assert all(m.isize == 100000 for m in ms)
    assert O.scan_members(parts[0]) == []


def test_stream_semantics():
    p = W.content(W.MARKOV, 1, 50000)
    c = W.gzip_member(p, 6).tobytes()
    assert O.decompress(b"")[0] == O.NOT_GZIP
    assert O.decompress(b"hello world")[0] == O.NOT_GZIP
    st, out = O.decompress(c + c)
    assert st == O.OK and out.tobytes() == p.tobytes() * 2
    st, out = O.decompress(c + b"trailing garbage bytes!!")
    assert st == O.OK and out.tobytes() == p.tobytes()
    assert O.decompress(c[:-20])[0] != O.OK
    bad = bytearray(c)
    bad[-8] ^= 1
    assert O.decompress(bytes(bad))[0] == O.CRC_MISMATCH
    bad = bytearray(c)
    bad[-4] ^= 1
    assert O.decompress(bytes(bad))[0] == O.SIZE_MISMATCH
    for blob in (c + c, c + b"trailing garbage bytes!!"):
        st, out, _ = O.decompress_chunked(blob, chunk_bytes=8192, threads=2)
        assert st == O.OK


def test_find_starts_keeps_true_stored_starts():
    """The partition-start rule (orc_find_starts): a stored candidate needs a
    stored or dynamic block right after it.  Its candidates are a subset of
    the reference's (orc_find_blocks), every true stored block start whose
    successor is stored or dynamic stays, and the false LEN/NLEN matches
    inside stored random bytes go."""
    import numpy as np
    from gzippy_b200 import workloads as W
    p = np.concatenate([W.content(k % 4, 60 + k, 1 << 20) for k in range(4)])
    for level in (0, 6):
        c = W.gzip_member(p, level)
        blocks = O.block_starts(c, p.size)
        bits = [b for b, _ in blocks]
        a = np.concatenate([c, np.zeros(2, np.uint8)])

        def btype(bit):
            return ((int(a[bit // 8]) >> (bit % 8) | int(a[bit // 8 + 1]) << (8 - bit % 8)) >> 1) & 3

        _, hl = O.gzip_header_len(c)
        f_all, s_all = O.find_blocks(c, hl * 8, c.size * 8, cap=1 << 20)
        f_st, s_st = O.find_starts(c, hl * 8, c.size * 8, cap=1 << 20)
        ref = set(zip(f_all.tolist(), s_all.tolist()))
        got = set(zip(f_st.tolist(), s_st.tolist()))
        assert got <= ref
        true_set = set(bits)
        for k in range(1, len(bits) - 1):
            b = bits[k]
            if btype(b) != 0 or btype(bits[k + 1]) not in (0, 2):
                continue
            bfinal = (int(a[b // 8]) >> (b % 8)) & 1
            # a non-final stored block with a non-empty LEN is a candidate
            off = (b + 3 + 7) // 8
            length = int(a[off]) | int(a[off + 1]) << 8
            if bfinal or length == 0:
                continue
            assert any(lo <= b <= hi for lo, hi in got), (level, b)
        false_ref = [x for x in ref if not any(x[0] <= t <= x[1] for t in true_set)]
        false_got = [x for x in got if not any(x[0] <= t <= x[1] for t in true_set)]
        assert len(false_got) <= len(false_ref) and len(false_got) <= 1, (level, len(false_ref), len(false_got))


def planted_false_stored_start(seed: int = 11):
    """A level-0 member (stored blocks only) of Markov text whose payload
    holds a planted false stored start: a byte below 0x20 (three zero header
    bits), LEN/NLEN, LEN bytes, then a second LEN/NLEN pair where the
    successor would sit.  Returns (compressed, plaintext, planted byte offset
    of the false LEN field in the compressed stream)."""
    text = bytearray(W.content(W.MARKOV, seed, 300_000).tobytes())
    plant = bytes([0x00, 0x10, 0x00, 0xEF, 0xFF]) + b"A" * 16 + bytes([0x00, 0x08, 0x00, 0xF7, 0xFF])
    at = 150_003
    text[at:at + len(plant)] = plant
    comp = W.gzip_member(np.frombuffer(bytes(text), np.uint8), 0)
    off = comp.tobytes().find(plant)
    assert off > 0
    return comp, bytes(text), off + 1


def test_planted_false_stored_start_is_repaired():
    """The stored start rule is a heuristic: a planted LEN/NLEN pair followed
    by a second one passes it.  The partition holding the plant takes it as
    its start, and the chain walk still returns the exact plaintext."""
    comp, plain, len_off = planted_false_stored_start()
    chunk = 4096
    _, hl = O.gzip_header_len(comp)
    b0 = hl * 8
    part = (len_off * 8 - b0) // (chunk * 8)
    lo, hi = b0 + part * chunk * 8, b0 + (part + 1) * chunk * 8
    first, seek = O.find_starts(comp, lo, hi)
    assert len(first) and int(seek[0]) == len_off * 8 - 3, "the plant is the partition's start"
    st, out, stats = O.decompress_chunked(comp, chunk_bytes=chunk, threads=4)
    assert st == O.OK and out.tobytes() == plain
    assert stats.n_spec_rejected + stats.n_repairs >= 1
