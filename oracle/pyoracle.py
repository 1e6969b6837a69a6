"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference arm are the only callers.  The product path never
imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "gzoracle.c")

OK, NOT_GZIP, BAD_HEADER, BAD_DEFLATE, CRC_MISMATCH, SIZE_MISMATCH, OUT_TOO_SMALL = range(7)
TRUNCATED = 9
WIN_MARKERS, WIN_BYTES = 0, 1

_lock = threading.Lock()
_lib = None


class ChunkResult(ctypes.Structure):
    _fields_ = [("end_bit", ctypes.c_uint64), ("out_len", ctypes.c_uint64),
                ("marker_end", ctypes.c_uint64), ("n_blocks", ctypes.c_uint32),
                ("n_stored", ctypes.c_uint32), ("n_fixed", ctypes.c_uint32),
                ("n_dynamic", ctypes.c_uint32), ("final_block", ctypes.c_int32),
                ("status", ctypes.c_int32)]


class Member(ctypes.Structure):
    _fields_ = [("start", ctypes.c_uint64), ("length", ctypes.c_uint64),
                ("deflate_start", ctypes.c_uint64), ("isize", ctypes.c_uint32),
                ("pad", ctypes.c_uint32), ("output_offset", ctypes.c_uint64)]


class ChunkedStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("n_chunks", "n_candidates_ok", "n_spec_rejected", "n_repairs",
                 "n_tail_marker_chunks", "n_members")]


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "gzoracle.h"))):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", LIB, SRC, "-lpthread"])
    return LIB


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(LIB)
            vp, sz, u64, u32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint32
            L.orc_crc32.argtypes = [u32, vp, sz]
            L.orc_crc32.restype = u32
            L.orc_crc32_combine.argtypes = [u32, u32, u64]
            L.orc_crc32_combine.restype = u32
            L.orc_gf2_mulmod.argtypes = [u32, u32]
            L.orc_gf2_mulmod.restype = u32
            L.orc_x_pow_8n.argtypes = [u64]
            L.orc_x_pow_8n.restype = u32
            L.orc_gzip_header.argtypes = [vp, sz, ctypes.POINTER(sz)]
            L.orc_find_blocks.argtypes = [vp, sz, u64, u64, vp, vp, sz]
            L.orc_find_blocks.restype = sz
            L.orc_find_starts.argtypes = [vp, sz, u64, u64, vp, vp, sz]
            L.orc_find_starts.restype = sz
            L.orc_is_dynamic_candidate.argtypes = [vp, sz, u64]
            L.orc_inflate_chunk.argtypes = [vp, sz, u64, u64, ctypes.c_int, vp, sz, vp, sz,
                                            ctypes.POINTER(ChunkResult)]
            L.orc_inflate_chunk_ex.argtypes = [vp, sz, u64, u64, ctypes.c_int, u64, vp, vp, sz, vp,
                                               sz, ctypes.POINTER(ChunkResult),
                                               ctypes.POINTER(ctypes.c_uint32),
                                               ctypes.POINTER(u64)]
            L.orc_fixed_sync_find.argtypes = [vp, sz, u64, u64, ctypes.POINTER(u64)]
            L.orc_dyn_sync_find.argtypes = [vp, sz, u64, u64, u64, ctypes.POINTER(u64)]
            L.orc_dynamic_lengths.argtypes = [vp, sz, u64, vp, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]
            L.orc_scan_members.argtypes = [vp, sz, vp, sz]
            L.orc_scan_members.restype = sz
            L.orc_decompress.argtypes = [vp, sz, vp, sz, ctypes.POINTER(sz)]
            L.orc_decompress_chunked.argtypes = [vp, sz, sz, ctypes.c_int, vp, sz,
                                                 ctypes.POINTER(sz), ctypes.POINTER(ChunkedStats)]
            _lib = L
    return _lib


def _u8(b) -> np.ndarray:
    if isinstance(b, np.ndarray):
        return np.ascontiguousarray(b, dtype=np.uint8)
    return np.frombuffer(bytes(b), dtype=np.uint8)


def crc32(data, crc: int = 0) -> int:
    a = _u8(data)
    return lib().orc_crc32(crc, a.ctypes.data, a.size)


def crc32_combine(c1: int, c2: int, len2: int) -> int:
    return lib().orc_crc32_combine(c1, c2, len2)


def gzip_header_len(data) -> tuple[int, int]:
    a = _u8(data)
    n = ctypes.c_size_t(0)
    st = lib().orc_gzip_header(a.ctypes.data, a.size, ctypes.byref(n))
    return st, n.value


def find_blocks(data, start_bit: int, end_bit: int, cap: int = 1 << 16):
    a = _u8(data)
    first = np.zeros(cap, np.uint64)
    seek = np.zeros(cap, np.uint64)
    k = lib().orc_find_blocks(a.ctypes.data, a.size, start_bit, end_bit,
                              first.ctypes.data, seek.ctypes.data, cap)
    k = min(k, cap)
    return first[:k].copy(), seek[:k].copy()


def find_starts(data, start_bit: int, end_bit: int, cap: int = 1 << 16):
    """find_blocks with the device's partition-start rule for stored
    candidates (the block after one is stored or a valid dynamic block)."""
    a = _u8(data)
    first = np.zeros(cap, np.uint64)
    seek = np.zeros(cap, np.uint64)
    k = lib().orc_find_starts(a.ctypes.data, a.size, start_bit, end_bit,
                              first.ctypes.data, seek.ctypes.data, cap)
    k = min(k, cap)
    return first[:k].copy(), seek[:k].copy()


def is_dynamic_candidate(data, bit: int) -> bool:
    a = _u8(data)
    return bool(lib().orc_is_dynamic_candidate(a.ctypes.data, a.size, bit))


def inflate_chunk(data, start_bit: int, stop_lo: int = 2**64 - 1, window=None,
                  markers: bool = False, cap: int | None = None):
    """Decode from start_bit to the first block boundary >= stop_lo (or the
    BFINAL block).  Returns (status, ChunkResult, u16 entries)."""
    a = _u8(data)
    cap = cap or max(1 << 16, a.size * 16)
    out = np.zeros(cap, np.uint16)
    res = ChunkResult()
    if window is not None:
        w = _u8(window)
        wp, wl = w.ctypes.data, w.size
    else:
        wp, wl = None, 0
    mode = WIN_MARKERS if markers else WIN_BYTES
    st = lib().orc_inflate_chunk(a.ctypes.data, a.size, start_bit, stop_lo, mode, wp, wl,
                                 out.ctypes.data, cap, ctypes.byref(res))
    return st, res, out[:res.out_len].copy()


def inflate_raw(data, cap: int | None = None):
    """A raw DEFLATE stream from bit 0 to its final block (the decode of
    decompress_raw_bytes, src/decompress/mod.rs:920), output capacity `cap`
    bytes.  Returns (status, bytes or None, end bit)."""
    a = _u8(data)
    st, res, out = inflate_chunk(a, 0, cap=cap or max(1 << 16, a.size * 16))
    ok = st == 0 and res.final_block
    return (st if not ok else 0), (out.astype(np.uint8).tobytes() if ok else None), res.end_bit


def block_starts(data, plain_len: int):
    """Every DEFLATE block of the single member `data` in stream order, as
    (absolute header bit, output offset at the block's start), by decoding
    one block at a time with the previous 32 KiB as window (the loop of
    scan_deflate, src/decompress/scan_inflate.rs:63-124).  plain_len is the
    member's output size."""
    a = _u8(data)
    st, hl = gzip_header_len(a)
    assert st == 0
    bit, out, win, blocks = hl * 8, 0, b"", []
    while True:
        blocks.append((bit, out))
        cap = min(plain_len - out + 64, 8 << 20)
        st, res, ent = inflate_chunk(a, bit, stop_lo=bit + 1, window=win, cap=cap)
        assert st == 0, st
        chunk = ent.astype(np.uint8).tobytes()
        win = (win + chunk)[-32768:]
        out += len(chunk)
        bit = res.end_bit
        if res.final_block:
            return blocks


def seek_index(data, plain: bytes, interval: int) -> bytes:
    """The seek index of a single-member gzip `data` whose output is `plain`:
    the checkpoint rule of scan_deflate (src/decompress/scan_inflate.rs:65-76)
    over block_starts, serialized in the version 1 layout load_index reads
    (src/decompress/index.rs:185-290): "GZIDX\\x01", deflate offset u32,
    output size u64, point count u32, 2 reserved bytes, then per point the
    bit offset from the deflate start u64, the output offset u64 and the
    32 KiB window.  No point qualifying gives one point at the start with a
    zero window (index.rs:124-134)."""
    import struct
    _, hl = gzip_header_len(data)
    pts, nxt = [], interval
    for bit, out in block_starts(data, len(plain)):
        if out >= nxt and out >= 32768:
            pts.append((bit - hl * 8, out))
            nxt = out + interval
    body = []
    if not pts:
        body.append(struct.pack("<QQ", 0, 0) + bytes(32768))
    for b, o in pts:
        body.append(struct.pack("<QQ", b, o) + plain[o - 32768:o])
    return (b"GZIDX\x01" + struct.pack("<IQIH", hl, len(plain), max(1, len(pts)), 0)
            + b"".join(body))


START_SYNC, ZERO_WINDOW = 1, 2


def inflate_chunk_ex(data, start_bit: int, stop_lo: int = 2**64 - 1, flags: int = 0,
                     start_table: int = 0, sync_targets=(), target_tables=None,
                     cap: int | None = None):
    """orc_inflate_chunk_ex: a chunk that may be a sync start (START_SYNC,
    inside the block whose header is at start_table; 0 = a fixed block) and
    stop at its successors' sync starts (target_tables: each one's block
    header, 0 = fixed).  Returns (status, ChunkResult, u16 entries, sync_end,
    end_hdr)."""
    a = _u8(data)
    cap = cap or max(1 << 16, a.size * 16)
    out = np.zeros(cap, np.uint16)
    res = ChunkResult()
    t = np.ascontiguousarray(sync_targets, dtype=np.uint64)
    tt = np.ascontiguousarray(target_tables if target_tables is not None else np.zeros(t.size),
                              dtype=np.uint64)
    se = ctypes.c_uint32(0)
    eh = ctypes.c_uint64(0)
    st = lib().orc_inflate_chunk_ex(a.ctypes.data, a.size, start_bit, stop_lo, flags, start_table,
                                    t.ctypes.data if t.size else None,
                                    tt.ctypes.data if t.size else None, t.size, out.ctypes.data,
                                    cap, ctypes.byref(res), ctypes.byref(se), ctypes.byref(eh))
    return st, res, out[:res.out_len].copy(), int(se.value), int(eh.value)


def dyn_sync_find(data, table_bit: int, from_bit: int, to_bit: int):
    """Sync start in the dynamic block whose header is at table_bit, or None."""
    a = _u8(data)
    b = ctypes.c_uint64(0)
    ok = lib().orc_dyn_sync_find(a.ctypes.data, a.size, table_bit, from_bit, to_bit, ctypes.byref(b))
    return int(b.value) if ok else None


def fixed_sync_find(data, from_bit: int, to_bit: int):
    """Sync start in fixed-Huffman data for [from_bit, to_bit), or None."""
    a = _u8(data)
    b = ctypes.c_uint64(0)
    ok = lib().orc_fixed_sync_find(a.ctypes.data, a.size, from_bit, to_bit, ctypes.byref(b))
    return int(b.value) if ok else None


def dynamic_lengths(data, bit: int):
    """(status, litlen lengths, dist lengths) of the dynamic header at `bit`."""
    a = _u8(data)
    lens = np.zeros(320, np.uint8)
    nl, nd = ctypes.c_int(0), ctypes.c_int(0)
    st = lib().orc_dynamic_lengths(a.ctypes.data, a.size, bit, lens.ctypes.data,
                                   ctypes.byref(nl), ctypes.byref(nd))
    return st, lens[:nl.value].copy(), lens[nl.value:nl.value + nd.value].copy()


def scan_members(data):
    a = _u8(data)
    k = lib().orc_scan_members(a.ctypes.data, a.size, None, 0)
    arr = (Member * max(k, 1))()
    if k:
        lib().orc_scan_members(a.ctypes.data, a.size, arr, k)
    return [arr[i] for i in range(k)]


def decompress(data, cap: int | None = None):
    """Serial whole-stream decode. Returns (status, bytes)."""
    a = _u8(data)
    cap = cap if cap is not None else max(1 << 20, a.size * 32)
    out = np.empty(max(cap, 1), np.uint8)
    n = ctypes.c_size_t(0)
    st = lib().orc_decompress(a.ctypes.data, a.size, out.ctypes.data, cap, ctypes.byref(n))
    return st, out[:n.value]


def decompress_chunked(data, chunk_bytes: int = 4 << 20, threads: int = 1,
                       cap: int | None = None):
    """Chunked speculative decode. Returns (status, bytes, stats)."""
    a = _u8(data)
    cap = cap if cap is not None else max(1 << 20, a.size * 32)
    out = np.empty(max(cap, 1), np.uint8)
    n = ctypes.c_size_t(0)
    stt = ChunkedStats()
    st = lib().orc_decompress_chunked(a.ctypes.data, a.size, chunk_bytes, threads,
                                      out.ctypes.data, cap, ctypes.byref(n), ctypes.byref(stt))
    return st, out[:n.value], stt
