"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Integer/byte work, so every comparison is bit-exact.  Kernel-level checks
compare the finder's candidate and each chunk's u16 entries (markers
included) with the oracle on the same inputs; end-to-end checks compare
whole streams with the oracle and with zlib."""
import io
import zlib

import numpy as np
import pytest

from oracle import pyoracle as O
from gzippy_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    import gzippy_b200 as G
    return G


# the Huffman block decoders: lane-parallel 32-bit steps, warp-uniform
# serial, lane-parallel 64-bit steps, chosen per block
DECODERS = [1, 2, 3, 4]
DECODER_IDS = ["steps", "serial", "wide", "adaptive"]


@pytest.fixture(scope="module", params=DECODERS, ids=DECODER_IDS)
def ctx(G, request):
    c = G.Context(chunk_bytes=32 << 10, decoder=request.param)
    yield c
    c.close()


# history layouts x decoders: (ring_history, decoder)
LAYOUTS = [(False, 1), (False, 2), (False, 3), (False, 4), (True, 0)]
LAYOUT_IDS = ["pages-steps", "pages-serial", "pages-wide", "pages-adaptive", "ring"]


def _stream(ctype, level, n, seed=1):
    p = W.content(ctype, seed, n)
    return p, W.gzip_member(p, level)


@pytest.mark.parametrize("ctype", [W.MARKOV, W.RANDOM, W.RUNS, W.RAMPS])
@pytest.mark.parametrize("level", [1, 6, 9])
def test_stream_matches_oracle_and_zlib(ctx, ctype, level):
    p, c = _stream(ctype, level, 700_000, seed=ctype * 10 + level)
    got = ctx.decompress(c)
    st, ref = O.decompress(c)
    assert st == O.OK
    assert got == ref.tobytes() == p.tobytes() == zlib.decompress(c.tobytes(), 31)


def _expected_start(data, f, t):
    """A partition's start: its first stored block start whose successor is a
    stored or dynamic block (searched first); else a sync start in
    fixed-Huffman data (searched next); else the first block-start
    candidate."""
    first, seek = O.find_starts(data, f, t, cap=1 << 18)
    a = np.concatenate([np.asarray(data, np.uint8), np.zeros(2, np.uint8)])
    for lo, hi in zip(first.tolist(), seek.tolist()):
        if (int(a[hi // 8]) >> (hi % 8) | int(a[hi // 8 + 1]) << (8 - hi % 8)) >> 1 & 3 == 0:
            return (int(lo), int(hi))              # BTYPE 00 at the start: stored
    b = O.fixed_sync_find(data, f, t)
    if b is not None:
        return ("sync", b)
    return (int(first[0]), int(seek[0])) if first.size else None


def test_finder_matches_oracle(ctx):
    p, c = _stream(W.MARKOV, 6, 2 << 20, seed=3)
    p2, c2 = _stream(W.RANDOM, 6, 1 << 20, seed=4)
    for data in (c, c2, np.concatenate([c, c2])):
        nbits = data.size * 8
        ranges = [(f, min(f + 64 * 1024 * 8, nbits)) for f in range(80, nbits, 97 * 1024 * 8 + 13)]
        got = ctx.debug_find(data, ranges)
        for (f, t), g in zip(ranges, got):
            exp = _expected_start(data, f, t)
            assert g == exp, (f, t, g, exp)


@pytest.mark.parametrize("layout", LAYOUTS, ids=LAYOUT_IDS)
def test_decode_chunks_match_oracle(G, layout):
    """Window-absent chunks from finder starts: entries, markers, end bits."""
    ring, dec = layout
    ctx = G.Context(chunk_bytes=32 << 10, ring_history=ring, decoder=dec)
    parts = [W.content(t, 5 + t, 1 << 20) for t in range(4)]
    plain = np.concatenate(parts)
    c = W.gzip_member(plain, 6)
    _, hl = O.gzip_header_len(c)
    nbits = c.size * 8
    starts, step = [], 40 * 1024 * 8
    for g in range(hl * 8 + step, nbits - 1000, step):
        first, seek = O.find_blocks(c, g, min(g + step, nbits), cap=4)
        if first.size:
            starts.append((int(first[0]), int(seek[0])))
    chunks = [(hl * 8, starts[0][0], True)]
    for k, (lo, hi) in enumerate(starts):
        stop = starts[k + 1][0] if k + 1 < len(starts) else 2**64 - 1
        chunks.append((hi, stop, False))
    cap = 4 << 20
    res, ent = ctx.debug_decode(c, chunks, cap)
    for i, (s, stop, mf) in enumerate(chunks):
        st, r, e = O.inflate_chunk(c, s, stop, markers=not mf, cap=cap)
        assert int(res[i, 4]) == st, i
        if st != O.OK:
            continue  # where an error is noticed is unspecified; the status must agree
        assert int(res[i, 0]) == r.end_bit and int(res[i, 1]) == r.out_len
        assert int(res[i, 2]) == r.marker_end and int(res[i, 5]) == r.final_block
        assert int(res[i, 3]) == r.n_blocks
        assert np.array_equal(ent[i, :r.out_len], e), i


@pytest.mark.parametrize("encoder", ["zlib-serial", "pigz"])
@pytest.mark.parametrize("layout", LAYOUTS, ids=LAYOUT_IDS)
def test_single_member_chunked_pipeline(G, layout, encoder):
    """One member of mixed content, as one serial deflate stream and in the
    pigz-style framing (an empty stored block every MiB)."""
    parts = [W.content(t % 4, 100 + t, 1 << 20) for t in range(12)]
    plain = np.concatenate(parts)
    c = W.encode_member(plain, 6, encoder, threads=4)
    ring, dec = layout
    for cb in (16 << 10, 64 << 10, 1 << 20):
        ctx = G.Context(chunk_bytes=cb, ring_history=ring, decoder=dec)
        got = ctx.decompress(c)
        s = ctx.stats()
        ctx.close()
        assert got == plain.tobytes(), cb
        assert s.n_accepted >= 1 and s.out_bytes == plain.size


def test_level1_fixed_blocks_repair_path(G):
    """No finder candidates inside fixed-Huffman data: the chain repairs."""
    p = W.content(W.MARKOV, 8, 1 << 20)
    c = W.gzip_member(p, 1)
    ctx = G.Context(chunk_bytes=16 << 10)
    assert ctx.decompress(c) == p.tobytes()
    ctx.close()


def test_multi_member(G, ctx):
    plains, comps = [], []
    for k in range(9):
        p, c = _stream(k % 4, [1, 6, 9][k % 3], 50_000 + 37_000 * k, seed=k)
        plains.append(p)
        comps.append(c)
    data = np.concatenate(comps)
    assert ctx.decompress(data) == np.concatenate(plains).tobytes()


def _zlib_members(data: bytes) -> bytes:
    out = []
    while data[:2] == b"\x1f\x8b":
        d = zlib.decompressobj(31)
        out.append(d.decompress(data))
        data = d.unused_data
    return b"".join(out)


def test_multi_member_segments_share_repair_passes(G):
    """Members walk as independent segments: the repairs of all members
    (level-1 fixed-Huffman members give the finder nothing to find) are
    decoded in a few shared passes, not one pass per member."""
    plains, comps = [], []
    for k in range(48):
        p, c = _stream(W.MARKOV if k % 2 else W.RAMPS, 1, 300_000 + 1111 * k, seed=100 + k)
        plains.append(p)
        comps.append(c)
    ctx = G.Context(chunk_bytes=16 << 10)
    assert ctx.decompress(np.concatenate(comps)) == np.concatenate(plains).tobytes()
    s = ctx.stats()
    assert s.n_members == 48
    assert s.decode_passes <= 8, s.decode_passes
    ctx.close()


def test_multi_member_false_member_plan_rewalks(G, ctx):
    """A member whose stored blocks carry a whole two-member gzip file: the
    scan plans members inside it, the segment before them ends elsewhere, and
    the stream is walked again as one segment."""
    inner = b"".join(_gz_level(W.content(W.MARKOV, 40 + k, 90_000).tobytes(), 6)
                     for k in range(2))
    outer_b = _gz_level(inner, 0)
    a = _gz_level(W.content(W.RAMPS, 43, 120_000).tobytes(), 6)
    c = _gz_level(W.content(W.RUNS, 44, 150_000).tobytes(), 9)
    data = a + outer_b + c
    want = _zlib_members(data)
    assert ctx.decompress(data) == want
    for cb in (8 << 10, 64 << 10):
        cx = G.Context(chunk_bytes=cb)
        assert cx.decompress(data) == want
        cx.close()


def _gz_level(data: bytes, level: int) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, 31)
    return c.compress(data) + c.flush()


def test_edge_cases(G, ctx):
    p, c = _stream(W.MARKOV, 6, 100_000, seed=2)
    cb = c.tobytes()
    empty = zlib.compressobj(6, zlib.DEFLATED, 31)
    e = empty.compress(b"") + empty.flush()
    assert ctx.decompress(b"") == b""
    assert ctx.decompress(b"\x1f") == b""
    assert ctx.decompress(b"not gzip at all") == b""
    assert ctx.decompress(e) == b""
    assert ctx.decompress(e + cb) == p.tobytes()
    assert ctx.decompress(cb + e + cb) == p.tobytes() * 2
    assert ctx.decompress(cb + b"trailing garbage!!!!!") == p.tobytes()
    tiny = zlib.compressobj(9, zlib.DEFLATED, 31)
    t = tiny.compress(b"a") + tiny.flush()
    assert ctx.decompress(t) == b"a"
    with pytest.raises(G.GzippyError):
        ctx.decompress(cb[:-30])
    bad = bytearray(cb)
    bad[-8] ^= 0x40
    with pytest.raises(G.GzippyError) as ei:
        ctx.decompress(bytes(bad))
    assert ei.value.code == G.CRC_MISMATCH
    bad = bytearray(cb)
    bad[-2] ^= 1
    with pytest.raises(G.GzippyError) as ei:
        ctx.decompress(bytes(bad))
    assert ei.value.code == G.SIZE_MISMATCH
    bad = bytearray(cb)
    bad[len(cb) // 2] ^= 0xFF
    with pytest.raises(G.GzippyError):
        ctx.decompress(bytes(bad))


def test_header_fields(G, ctx):
    """FTEXT/FHCRC/FEXTRA/FNAME/FCOMMENT members (RFC 1952 2.3.1)."""
    p = W.content(W.RAMPS, 4, 200_000).tobytes()
    raw = zlib.compressobj(6, zlib.DEFLATED, -15)
    body = raw.compress(p) + raw.flush()
    trailer = zlib.crc32(p).to_bytes(4, "little") + len(p).to_bytes(4, "little")
    hdr = bytes([0x1f, 0x8b, 8, 0x1f, 0, 0, 0, 0, 0, 3]) + (6).to_bytes(2, "little") + b"XYZ\x00\x01\x02"
    hdr += b"name.txt\x00" + b"a comment\x00"
    hdr += (zlib.crc32(hdr) & 0xFFFF).to_bytes(2, "little")
    data = hdr + body + trailer
    assert ctx.decompress(data) == p
    assert O.decompress(data)[1].tobytes() == p


def test_writer_api(G, ctx):
    p, c = _stream(W.RUNS, 6, 3 << 20, seed=7)
    buf = io.BytesIO()
    n = ctx.decompress_to_writer(c, buf)
    assert n == p.size and buf.getvalue() == p.tobytes()
    assert G.decompress_to_writer(b"xx", io.BytesIO()) == 0


def test_batch_matches_individual(G, ctx):
    rng = np.random.default_rng(0)
    datas, plains = [], []
    for i in range(60):
        n = int(rng.integers(0, 300_000))
        p, c = _stream(int(rng.integers(0, 4)), int(rng.choice([1, 6, 9])), n, seed=100 + i)
        datas.append(c.tobytes())
        plains.append(p.tobytes())
    datas.append(b"not gzip")
    plains.append(b"")
    bad = bytearray(datas[3])
    bad[-8] ^= 1
    datas.append(bytes(bad))
    res = ctx.decompress_batch(datas)
    for i in range(61):
        assert res[i] == plains[i], i
    assert isinstance(res[61], G.GzippyError)


def _pack16(blobs):
    offs, at = [], 0
    for b in blobs:
        offs.append(at)
        at += (len(b) + 15) & ~15
    buf = np.zeros(at + 1024, np.uint8)
    for o, b in zip(offs, blobs):
        buf[o:o + len(b)] = np.frombuffer(b, np.uint8)
    return buf, np.array(offs, np.uint64), np.array([len(b) for b in blobs], np.uint64)


def test_batch_device_matches_individual(G, ctx):
    """Device-resident batch: every stream's slice of the packed output equals
    its own decode; failing and non-gzip streams report their status."""
    import torch
    rng = np.random.default_rng(7)
    blobs, want = [], []
    for k in range(60):
        n = int(rng.integers(1, 400_000))
        p, c = _stream(k % 4, [1, 6, 9][k % 3], n, seed=200 + k)
        blobs.append(c.tobytes())
        want.append(p.tobytes())
    blobs.append(blobs[3] + blobs[4])           # two members
    want.append(want[3] + want[4])
    blobs.append(b"not gzip")
    want.append(b"")
    blobs.append(_gz_level(b"", 6))
    want.append(b"")
    bad = bytearray(blobs[5])
    bad[-8] ^= 1                                 # CRC mismatch
    blobs.append(bytes(bad))
    want.append(None)
    buf, offs, lens = _pack16(blobs)
    d_in = torch.from_numpy(buf).cuda()
    cap = sum(len(w) for w in want if w) + 4096
    d_out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    with pytest.raises(G.GzippyError) as ei:
        ctx.decompress_batch_device(d_in.data_ptr(), offs, lens, d_out.data_ptr(), cap)
    assert ei.value.code == G.CRC_MISMATCH
    good = [i for i, w in enumerate(want) if w is not None]
    blobs_g = [blobs[i] for i in good]
    buf, offs, lens = _pack16(blobs_g)
    d_in = torch.from_numpy(buf).cuda()
    oo, ol, st = ctx.decompress_batch_device(d_in.data_ptr(), offs, lens, d_out.data_ptr(), cap)
    host = d_out.cpu().numpy()
    for j, i in enumerate(good):
        assert st[j] == (G.NOT_GZIP if blobs[i] == b"not gzip" else G.OK)
        assert host[int(oo[j]):int(oo[j]) + int(ol[j])].tobytes() == want[i], i
    with pytest.raises(G.GzippyError) as ei:
        ctx.decompress_batch_device(d_in.data_ptr(), offs, lens, d_out.data_ptr(), 100)
    assert ei.value.code == G.OUT_TOO_SMALL


def test_autotune_caches_per_kind(G):
    """The first job of a kind runs the tuning trials, the next reuses the
    choice; every trial's output is byte-exact."""
    p, c = _stream(W.MARKOV, 6, 3 << 20, seed=31)
    cx = G.Context(autotune=1)
    assert cx.decompress(c) == p.tobytes()
    s1 = cx.stats()
    assert s1.tune_trials >= 4 and s1.tune_key != 0
    assert s1.chunk_bytes in (16 << 10, 32 << 10, 64 << 10, 128 << 10)
    assert s1.lut_bits in (10, 11, 12) and s1.ctas_per_sm in (3, 4)
    assert cx.decompress(c) == p.tobytes()
    s2 = cx.stats()
    assert s2.tune_trials == 0 and s2.tune_key == s1.tune_key
    assert (s2.chunk_bytes, s2.lut_bits, s2.ctas_per_sm) == (s1.chunk_bytes, s1.lut_bits, s1.ctas_per_sm)
    cx.close()


def _level1(ctype, n, seed):
    p = W.content(ctype, seed, n)
    return p, W.gzip_member(p, 1)   # level 1 = fixed-Huffman blocks (stored for random bytes)


def test_sync_find_matches_oracle(ctx):
    """Partitions get the oracle's sync start in fixed-Huffman data, searched
    first, or else its first block-start candidate."""
    for ctype, seed in ((W.MARKOV, 41), (W.RUNS, 42), (W.RAMPS, 43)):
        p, c = _level1(ctype, 3 << 20, seed)
        nbits = c.size * 8
        ranges = [(f, min(f + 40 * 1024 * 8, nbits)) for f in range(200, nbits, 37 * 1024 * 8 + 5)]
        got = ctx.debug_find(c, ranges)
        n_sync = 0
        for (f, t), g in zip(ranges, got):
            exp = _expected_start(c, f, t)
            n_sync += exp is not None and exp[0] == "sync"
            assert g == exp, (ctype, f, t, g, exp)
        if ctype != W.RAMPS:
            assert n_sync > len(ranges) // 2


def test_sync_chunks_match_oracle(G, ctx):
    """Chunks that start at sync starts (mid-block, fixed table) and chunks
    that stop at them: entries, end bits and sync_end equal the oracle's,
    including a bogus sync start that the predecessor goes by."""
    p, c = _level1(W.MARKOV, 2 << 20, 44)
    _, hl = O.gzip_header_len(c)
    nbits = c.size * 8
    step = 40 * 1024 * 8
    syncs = [O.fixed_sync_find(c, g, g + step) for g in range(hl * 8 + step, nbits - step, step)]
    syncs = [b for b in syncs if b is not None]
    assert len(syncs) >= 4
    starts = syncs[:2] + [syncs[2] + 1] + syncs[2:]          # a bogus one before a true one
    chunks = [(hl * 8, starts[0], 1)] + [
        (s, starts[k + 1] if k + 1 < len(starts) else 2**64 - 1, 2) for k, s in enumerate(starts)]
    cap = 4 << 20
    res, ent = ctx.debug_decode(c, chunks, cap)
    n_synced = 0
    for i, (s, stop, fl) in enumerate(chunks):
        targets = starts[i:i + 5]                             # successors: all sync starts
        st, r, e, se, _ = O.inflate_chunk_ex(c, s, stop, flags=(O.START_SYNC if fl & 2 else O.ZERO_WINDOW),
                                             sync_targets=targets, cap=cap)
        assert int(res[i, 4]) == st, i
        if st != O.OK:
            continue
        assert int(res[i, 0]) == r.end_bit and int(res[i, 1]) == r.out_len, i
        assert int(res[i, 2]) == r.marker_end and int(res[i, 5]) == r.final_block, i
        assert int(res[i, 3]) == r.n_blocks and int(res[i, 6]) == se, i
        assert np.array_equal(ent[i, :r.out_len], e), i
        n_synced += se
    assert n_synced >= 3


def test_level1_fixed_streams_split(G):
    """Fixed-Huffman members decode in many accepted chunks, byte-exact."""
    for ctype in (W.MARKOV, W.RUNS):
        p, c = _level1(ctype, 6 << 20, 45 + ctype)
        cx = G.Context(chunk_bytes=32 << 10)
        assert cx.decompress(c) == p.tobytes()
        s = cx.stats()
        d, r = cx.last_chunks()
        assert s.n_accepted >= 8, (ctype, s.n_accepted)
        assert int(((d["flags"] & 8) != 0).sum()) >= 4
        assert int(r["sync_end"].sum()) >= 4
        cx.close()


def _first_block(c):
    _, hl = O.gzip_header_len(c)
    h = hl * 8
    st, r, _ = O.inflate_chunk(c, h, stop_lo=h + 1, cap=16 << 20)
    assert st == O.OK
    return h, r.end_bit


def test_dyn_sync_find_matches_oracle(ctx):
    """Sync starts inside a dynamic block equal the oracle's."""
    for ctype, seed in ((W.RUNS, 51), (W.MARKOV, 52), (W.RAMPS, 53)):
        p, c = _stream(ctype, 6, 3 << 20, seed=seed)
        h, end = _first_block(c)
        items = [(h, g, g + 40000) for g in range(h + 3000, end - 40000, 17000)]
        got = ctx.debug_dyn_sync(c, items)
        exp = [O.dyn_sync_find(c, t, f, e) for t, f, e in items]
        assert got == exp, (ctype, got, exp)
        if ctype != W.RAMPS:
            assert sum(x is not None for x in got) >= len(items) // 2


def test_dyn_sync_chunks_match_oracle(ctx):
    """A dynamic block cut at sync starts: entries, end bits, sync ends and
    end headers equal the oracle's, and a bogus sync start is gone by."""
    p, c = _stream(W.RUNS, 6, 3 << 20, seed=54)
    h, end = _first_block(c)
    syncs = [O.dyn_sync_find(c, h, g, g + 40000) for g in range(h + 3000, end - 40000, 40000)]
    syncs = [b for b in syncs if b is not None][:4]
    assert len(syncs) >= 3
    starts = [syncs[0], syncs[1] + 1, syncs[1]] + syncs[2:]
    starts = sorted(set(starts))
    chunks = [(h, starts[0], 1)] + [(s, starts[k + 1] if k + 1 < len(starts) else 2**64 - 1, 2)
                                     for k, s in enumerate(starts)]
    tables = [0] + [h] * len(starts)
    cap = 8 << 20
    res, ent = ctx.debug_decode(c, chunks, cap, tables=tables)
    n_synced = 0
    for i, (s, stop, fl) in enumerate(chunks):
        tg = starts[i:i + 5]
        st, r, e, se, eh = O.inflate_chunk_ex(
            c, s, stop, flags=(O.START_SYNC if fl & 2 else O.ZERO_WINDOW),
            start_table=(h if fl & 2 else 0), sync_targets=tg, target_tables=[h] * len(tg), cap=cap)
        assert int(res[i, 4]) == st, i
        if st != O.OK:
            continue
        assert int(res[i, 0]) == r.end_bit and int(res[i, 1]) == r.out_len, i
        assert int(res[i, 2]) == r.marker_end and int(res[i, 5]) == r.final_block, i
        assert int(res[i, 3]) == r.n_blocks and int(res[i, 6]) == se, i
        assert np.array_equal(ent[i, :r.out_len], e), i
        n_synced += se
    assert n_synced >= 2


def test_high_ratio_partitions_split_at_dyn_sync(G):
    """Byte runs (about 15x) with fine_split: partitions are cut by their
    output estimate and the pieces start at sync starts inside dynamic
    blocks; byte-exact."""
    p, c = _stream(W.RUNS, 6, 24 << 20, seed=55)
    cx = G.Context(chunk_bytes=64 << 10, fine_split=True)
    assert cx.decompress(c) == p.tobytes()
    d, r = cx.last_chunks()
    dyn = ((d["flags"] & 8) != 0) & (d["table_bit"] != 0)
    assert int(dyn.sum()) >= 4
    assert int((r["sync_end"][:len(d)] != 0).sum()) >= 4
    cx.close()


def test_sync_start_naming_a_fixed_block_header(ctx):
    """A sync start may name its block's header when that block is fixed (a
    repair after a mid-block handover does): same entries as the oracle."""
    p, c = _level1(W.MARKOV, 1 << 20, 56)
    h, end = _first_block(c)
    b = O.fixed_sync_find(c, h + 2000, end)
    assert b is not None
    res, ent = ctx.debug_decode(c, [(b, 2**64 - 1, 2)], 4 << 20, tables=[h])
    st, r, e, se, _ = O.inflate_chunk_ex(c, b, flags=O.START_SYNC, start_table=h, cap=4 << 20)
    assert st == O.OK and int(res[0, 4]) == st
    assert int(res[0, 0]) == r.end_bit and int(res[0, 1]) == r.out_len
    assert np.array_equal(ent[0, :r.out_len], e)


def test_planted_false_stored_start(G, ctx):
    """A stored-block payload that holds a LEN/NLEN pair followed by a second
    one passes the stored start rule: the finder takes it as its partition's
    start (like the oracle) and the chain walk still returns the exact
    plaintext."""
    from test_oracle import planted_false_stored_start
    comp, plain, len_off = planted_false_stored_start()
    f = len_off * 8 - 2000
    got = ctx.debug_find(comp, [(f, f + 8000)])
    assert got[0] == _expected_start(comp, f, f + 8000)
    assert got[0][1] == len_off * 8 - 3
    for cb in (16 << 10, 32 << 10):
        c2 = G.Context(chunk_bytes=cb)
        assert c2.decompress(comp) == plain
        c2.close()
