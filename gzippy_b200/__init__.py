"""gzippy_b200 -- B200 (sm_100a) gzip decompression behind gzippy's API.

Mirrors the reference's public decode API (JackDanger/gzippy v0.8.0,
src/lib.rs:176-227):

    decompress(data) -> bytes
    decompress_with_threads(data, threads) -> bytes
    decompress_to_writer(data, writer) -> int
    decompress_to_writer_with_threads(data, writer, threads) -> int

Non-gzip input returns b"" / 0 (src/lib.rs:50-52).  Corrupt or truncated
input raises GzippyError (kind "Decompression", src/error.rs:7-46).  The
thread count of the reference has no meaning on the device; it is accepted
and ignored.  Every call goes through the C ABI of libgzgpu.so
(include/gzgpu.h); there is no CPU fallback: without the CUDA library or a
CUDA device the calls raise.

Beyond the reference: decompress_batch (many streams per launch) and
Server (continuous-batching request loop).
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from . import build as _build

__all__ = ["GzippyError", "decompress", "decompress_with_threads", "decompress_to_writer",
           "decompress_to_writer_with_threads", "decompress_batch", "Context", "Server", "Stats",
           "lib"]

OK, NOT_GZIP, BAD_HEADER, BAD_DEFLATE, CRC_MISMATCH, SIZE_MISMATCH, OUT_TOO_SMALL = range(7)
DEVICE_ERROR, TIMEOUT, TRUNCATED, INVALID_ARGUMENT = 7, 8, 9, 12
NOALLOC_TOO_LARGE = 14
OVER_BUDGET, PENDING = 15, 16
NOALLOC_MAX_OUT = 4 << 20


class GzippyError(Exception):
    """gzippy's GzippyError; `kind` is the variant name, `code` the C status."""

    def __init__(self, kind: str, message: str, code: int = 0):
        super().__init__(f"{kind} error: {message}")
        self.kind = kind
        self.code = code


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("chunk_bytes", ctypes.c_size_t),
                ("lut_bits", ctypes.c_int), ("autotune", ctypes.c_int),
                ("ring_history", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("fine_split", ctypes.c_int), ("high_priority", ctypes.c_int),
                ("work_order", ctypes.c_int), ("decoder", ctypes.c_int)]


class Span(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("len", ctypes.c_size_t)]


class Out(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("cap", ctypes.c_size_t), ("len", ctypes.c_size_t)]


class Stats(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in
                 ("ms_total", "ms_h2d", "ms_scan", "ms_find", "ms_decode", "ms_walk",
                  "ms_resolve", "ms_crc", "ms_d2h", "ms_decode_kernel")] +
                [(n, ctypes.c_uint64) for n in
                 ("in_bytes", "out_bytes", "n_streams", "n_members", "n_chunks", "n_accepted",
                  "n_rejected", "n_repairs", "n_tail_marker_chunks", "n_pages", "decode_passes",
                  "kernel_launches", "chunk_bytes")] +
                [("lut_bits", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32),
                 ("tune_key", ctypes.c_uint32), ("tune_trials", ctypes.c_uint32),
                 ("pool_regrows", ctypes.c_uint32), ("reserved", ctypes.c_uint32)])

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("lanes", ctypes.c_int), ("autotune", ctypes.c_int),
                ("small_lanes", ctypes.c_int), ("budget_bytes", ctypes.c_size_t),
                ("max_batch_bytes", ctypes.c_size_t), ("max_batch_requests", ctypes.c_size_t),
                ("large_bytes", ctypes.c_size_t)]


class RequestTimes(ctypes.Structure):
    _fields_ = [("queue_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("submitted", "completed", "batches", "in_flight", "queued", "budget_used",
                 "in_bytes", "out_bytes")]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


WRITE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)

_lock = threading.Lock()
_lib = None
_default_ctx = None


def lib():
    """The loaded libgzgpu.so (built in-tree on first use if missing)."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.LIB
            if not os.path.exists(path):
                _build.build()
            L = ctypes.CDLL(path)
            vp, sz = ctypes.c_void_p, ctypes.c_size_t
            L.gzgpu_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(Config)]
            L.gzgpu_destroy.argtypes = [vp]
            L.gzgpu_strerror.argtypes = [ctypes.c_int]
            L.gzgpu_strerror.restype = ctypes.c_char_p
            L.gzgpu_decompress.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(sz)]
            L.gzgpu_decompress_device.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(sz)]
            L.gzgpu_inflate_raw.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(sz)]
            L.gzgpu_inflate_zlib.argtypes = [vp, vp, sz, vp, sz, ctypes.POINTER(sz)]
            L.gzgpu_build_index.argtypes = [vp, vp, sz, ctypes.c_uint64, vp, sz, ctypes.POINTER(sz)]
            L.gzgpu_decompress_to_writer.argtypes = [vp, vp, sz, WRITE_FN, vp,
                                                     ctypes.POINTER(ctypes.c_uint64)]
            u64p = ctypes.POINTER(ctypes.c_uint64)
            L.gzgpu_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ServerConfig)]
            L.gzgpu_server_destroy.argtypes = [vp]
            L.gzgpu_server_destroy.restype = None
            L.gzgpu_submit.argtypes = [vp, vp, sz, vp, sz, u64p]
            L.gzgpu_poll.argtypes = [vp, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(sz),
                                     ctypes.POINTER(RequestTimes)]
            L.gzgpu_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
            L.gzgpu_decompress_batch_device.argtypes = [vp, vp, u64p, u64p, sz, vp, sz, u64p, u64p,
                                                        ctypes.POINTER(ctypes.c_int)]
            L.gzgpu_decompress_batch.argtypes = [vp, ctypes.POINTER(Span), sz, ctypes.POINTER(Out),
                                                 ctypes.POINTER(ctypes.c_int)]
            L.gzgpu_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
            L.gzgpu_debug_find.argtypes = [vp, vp, sz, vp, vp, sz, vp, vp, vp]
            L.gzgpu_debug_decode.argtypes = [vp, vp, sz, vp, vp, vp, sz, vp, sz, vp, vp]
            L.gzgpu_debug_dyn_sync.argtypes = [vp, vp, sz, vp, vp, vp, sz, vp, vp]
            L.gzgpu_debug_last_chunks.argtypes = [vp, vp, vp, sz, ctypes.POINTER(sz)]
            L.gzgpu_decompress_device_noalloc.argtypes = [vp, sz, vp, sz, ctypes.POINTER(sz), vp]
            _lib = L
    return _lib


def strerror(code: int) -> str:
    return lib().gzgpu_strerror(code).decode()


def _raise(code: int):
    if code == TRUNCATED:
        raise GzippyError("Decompression", strerror(code), code)
    if code == INVALID_ARGUMENT:
        raise GzippyError("InvalidArgument", strerror(code), code)
    raise GzippyError("Decompression", strerror(code), code)


def _as_u8(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data.reshape(-1).view(np.uint8))
    return np.frombuffer(memoryview(data).cast("B"), dtype=np.uint8)


class Context:
    """One device context (gzgpu_ctx): device buffers, stream, statistics."""

    def __init__(self, device: int = 0, chunk_bytes: int = 0, lut_bits: int = 0,
                 autotune: bool = False, ring_history: bool = False, ctas_per_sm: int = 0,
                 fine_split: bool = False, high_priority: bool = False,
                 longest_first: bool = True, decoder: int = 0):
        self._lib = lib()
        cfg = Config(device, chunk_bytes, lut_bits, int(autotune), int(ring_history), ctas_per_sm,
                     int(fine_split), int(high_priority), 0 if longest_first else 1, decoder)
        h = ctypes.c_void_p()
        rc = self._lib.gzgpu_create(ctypes.byref(h), ctypes.byref(cfg))
        if rc != OK:
            raise GzippyError("Internal", f"gzgpu_create: {strerror(rc)}", rc)
        self._h = h
        self._hint = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.gzgpu_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def stats(self) -> Stats:
        s = Stats()
        self._lib.gzgpu_get_stats(self._h, ctypes.byref(s))
        return s

    def decompress_into(self, data, out: np.ndarray) -> int:
        """Decode into a caller buffer; returns bytes written; raises on error."""
        a = _as_u8(data)
        n = ctypes.c_size_t(0)
        rc = self._lib.gzgpu_decompress(self._h, a.ctypes.data, a.size, out.ctypes.data,
                                        out.size, ctypes.byref(n))
        if rc == NOT_GZIP:
            return 0
        if rc != OK:
            if rc == OUT_TOO_SMALL:
                raise GzippyError("Decompression", f"output needs {n.value} bytes", rc)
            _raise(rc)
        return n.value

    def decompress(self, data) -> bytes:
        a = _as_u8(data)
        cap = max(self._hint, a.size * 4 + 4096)
        for _ in range(3):
            out = np.empty(cap, dtype=np.uint8)
            n = ctypes.c_size_t(0)
            rc = self._lib.gzgpu_decompress(self._h, a.ctypes.data, a.size, out.ctypes.data, cap,
                                            ctypes.byref(n))
            if rc == NOT_GZIP:
                return b""
            if rc == OUT_TOO_SMALL:
                cap = n.value
                continue
            if rc != OK:
                _raise(rc)
            return out[:n.value].tobytes()
        _raise(OUT_TOO_SMALL)

    def inflate_raw(self, data, _entry: str = "gzgpu_inflate_raw") -> bytes:
        """One raw DEFLATE stream (gzippy::decompress_raw, src/lib.rs:250):
        decoded up to its final block, trailing bytes ignored; raises on
        invalid or cut-off data.  The first output guess is 4x the input, as
        in decompress_raw_bytes (src/decompress/mod.rs:920); a short guess is
        retried once at the exact size."""
        a = _as_u8(data)
        cap = max(4096, a.size * 4)
        fn = getattr(self._lib, _entry)
        for _ in range(2):
            out = np.empty(cap, dtype=np.uint8)
            n = ctypes.c_size_t(0)
            rc = fn(self._h, a.ctypes.data, a.size, out.ctypes.data, cap, ctypes.byref(n))
            if rc == OUT_TOO_SMALL:
                cap = n.value
                continue
            if rc != OK:
                _raise(rc)
            return out[:n.value].tobytes()
        _raise(OUT_TOO_SMALL)

    def inflate_zlib(self, data) -> bytes:
        """zlib data (decompress_zlib_turbo, src/decompress/mod.rs:895): the
        DEFLATE stream between the 2-byte header and the Adler-32 trailer,
        neither checked, as in the reference."""
        if len(data) < 6:
            _raise(INVALID_ARGUMENT)
        return self.inflate_raw(data, "gzgpu_inflate_zlib")

    def build_index(self, data, interval_bytes: int = 1 << 20) -> bytes:
        """gzippy's seek index of a single-member gzip buffer (build_index +
        serialize_index, src/decompress/index.rs:55-141), version 1 layout.
        Sized from the member's ISIZE; a short guess (ISIZE wraps past
        4 GiB) is retried at the exact size."""
        a = _as_u8(data)
        isize = int(a[-4:].view("<u4")[0]) if a.size >= 4 else 0
        pts = isize // max(interval_bytes, 1) + 2 if interval_bytes else isize // 1024 + 2
        cap = 24 + pts * (16 + 32768)
        for _ in range(2):
            out = np.empty(cap, dtype=np.uint8)
            n = ctypes.c_size_t(0)
            rc = self._lib.gzgpu_build_index(self._h, a.ctypes.data, a.size, interval_bytes,
                                             out.ctypes.data, cap, ctypes.byref(n))
            if rc == OUT_TOO_SMALL:
                cap = n.value
                continue
            if rc != OK:
                _raise(rc)
            return out[:n.value].tobytes()
        _raise(OUT_TOO_SMALL)

    def decompress_to_writer(self, data, writer) -> int:
        a = _as_u8(data)
        err = []

        def cb(_user, ptr, n):
            try:
                writer.write(ctypes.string_at(ptr, n))
                return 0
            except Exception as e:  # pragma: no cover
                err.append(e)
                return 1

        fn = WRITE_FN(cb)
        written = ctypes.c_uint64(0)
        rc = self._lib.gzgpu_decompress_to_writer(self._h, a.ctypes.data, a.size, fn, None,
                                                  ctypes.byref(written))
        if err:
            raise GzippyError("Io", str(err[0]))
        if rc == NOT_GZIP:
            return 0
        if rc != OK:
            _raise(rc)
        return written.value

    def decompress_device(self, d_in: int, in_len: int, d_out: int, out_cap: int) -> int:
        """Device-resident decode (raw device pointers); returns bytes written."""
        n = ctypes.c_size_t(0)
        rc = self._lib.gzgpu_decompress_device(self._h, d_in, in_len, d_out, out_cap,
                                               ctypes.byref(n))
        if rc == NOT_GZIP:
            return 0
        if rc != OK:
            if rc == OUT_TOO_SMALL:
                raise GzippyError("Decompression", f"output needs {n.value} bytes", rc)
            _raise(rc)
        return n.value

    def decompress_batch_device(self, d_in: int, in_offs, in_lens, d_out: int, out_cap: int):
        """Many device-resident streams in one job (gzgpu_decompress_batch_device).
        Returns (out_offs, out_lens, statuses) as numpy arrays; raises on a
        failing stream or a too-small output."""
        offs = np.ascontiguousarray(in_offs, dtype=np.uint64)
        lens = np.ascontiguousarray(in_lens, dtype=np.uint64)
        n = offs.size
        oo = np.zeros(max(n, 1), np.uint64)
        ol = np.zeros(max(n, 1), np.uint64)
        st = np.zeros(max(n, 1), np.int32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        rc = self._lib.gzgpu_decompress_batch_device(
            self._h, d_in, offs.ctypes.data_as(u64p), lens.ctypes.data_as(u64p), n, d_out, out_cap,
            oo.ctypes.data_as(u64p), ol.ctypes.data_as(u64p),
            st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        if rc not in (OK, NOT_GZIP):
            if rc == OUT_TOO_SMALL:
                raise GzippyError("Decompression", f"output needs {int(ol[:n].sum())} bytes", rc)
            _raise(rc)
        return oo[:n], ol[:n], st[:n]

    def debug_find(self, data, ranges):
        """Finder kernel on explicit bit ranges -> list of (lo, hi) or None."""
        a = _as_u8(data)
        n = len(ranges)
        fr = np.array([r[0] for r in ranges], np.uint64)
        to = np.array([r[1] for r in ranges], np.uint64)
        lo = np.zeros(n, np.uint64)
        hi = np.zeros(n, np.uint64)
        va = np.zeros(n, np.int32)
        rc = self._lib.gzgpu_debug_find(self._h, a.ctypes.data, a.size, fr.ctypes.data,
                                        to.ctypes.data, n, lo.ctypes.data, hi.ctypes.data,
                                        va.ctypes.data)
        if rc != OK:
            _raise(rc)
        return [None if not va[i] else ((int(lo[i]), int(hi[i])) if va[i] == 1 else ("sync", int(lo[i])))
                for i in range(n)]

    def debug_dyn_sync(self, data, items):
        """Dynamic sync-start search on [(table_bit, from_bit, to_bit)] -> bit or None each."""
        a = _as_u8(data)
        n = len(items)
        tb = np.array([x[0] for x in items], np.uint64)
        fr = np.array([x[1] for x in items], np.uint64)
        to = np.array([x[2] for x in items], np.uint64)
        out = np.zeros(n, np.uint64)
        va = np.zeros(n, np.int32)
        rc = self._lib.gzgpu_debug_dyn_sync(self._h, a.ctypes.data, a.size, tb.ctypes.data,
                                            fr.ctypes.data, to.ctypes.data, n, out.ctypes.data,
                                            va.ctypes.data)
        if rc != OK:
            _raise(rc)
        return [int(out[i]) if va[i] else None for i in range(n)]

    def debug_decode(self, data, chunks, cap_per, tables=None):
        """Inflate kernel on explicit chunks [(start_bit, stop_bit, flags)], flags bit 0 =
        member start, bit 1 = sync start.  Returns (results n x 7 uint64: end_bit,
        out_len, marker_end, n_blocks, status, final_block, sync_end; entries n x
        cap_per uint16)."""
        a = _as_u8(data)
        n = len(chunks)
        st = np.array([c[0] for c in chunks], np.uint64)
        sp = np.array([c[1] for c in chunks], np.uint64)
        mf = np.array([int(c[2]) for c in chunks], np.int32)
        ent = np.zeros((n, cap_per), np.uint16)
        res = np.zeros((n, 7), np.uint64)
        tb = np.array(tables if tables is not None else [0] * n, np.uint64)
        rc = self._lib.gzgpu_debug_decode(self._h, a.ctypes.data, a.size, st.ctypes.data,
                                          sp.ctypes.data, mf.ctypes.data, n, ent.ctypes.data,
                                          cap_per, res.ctypes.data, tb.ctypes.data)
        if rc != OK:
            _raise(rc)
        return res, ent

    DESC_DTYPE = np.dtype([("start_bit", "<u8"), ("lo_bit", "<u8"), ("stop_lo", "<u8"),
                           ("guess_bit", "<u8"), ("limit_bit", "<u8"), ("in_end", "<u8"),
                           ("abort_bit", "<u8"), ("table_bit", "<u8"), ("flags", "<u4"),
                           ("stream", "<u4"), ("next", "<u4"), ("est_ratio", "<f4")])
    RESULT_DTYPE = np.dtype([("end_bit", "<u8"), ("out_len", "<u8"), ("marker_end", "<u8"),
                             ("last_page", "<u4"), ("prev_page", "<u4"), ("n_pages", "<u4"),
                             ("n_blocks", "<u4"), ("status", "<i4"), ("final_block", "<i4"),
                             ("t_start", "<u8"), ("t_end", "<u8"), ("gen", "<u4"),
                             ("sync_end", "<u4"), ("end_hdr_bit", "<u8")])

    def last_chunks(self):
        """(descs, results) structured arrays of the last job's chunk table."""
        n = ctypes.c_size_t(0)
        self._lib.gzgpu_debug_last_chunks(self._h, None, None, 0, ctypes.byref(n))
        d = np.zeros(n.value, self.DESC_DTYPE)
        r = np.zeros(n.value, self.RESULT_DTYPE)
        self._lib.gzgpu_debug_last_chunks(self._h, d.ctypes.data, r.ctypes.data, n.value,
                                          ctypes.byref(n))
        return d, r

    def decompress_batch(self, datas, caps=None):
        """Decode many streams in one job.  Returns a list of bytes (or a
        GzippyError instance per failed stream)."""
        arrs = [_as_u8(d) for d in datas]
        n = len(arrs)
        caps = caps or [max(a.size * 8 + 4096, 1 << 16) for a in arrs]
        for _ in range(3):
            outs_np = [np.empty(c, dtype=np.uint8) for c in caps]
            spans = (Span * max(n, 1))()
            outs = (Out * max(n, 1))()
            for i, (a, o) in enumerate(zip(arrs, outs_np)):
                spans[i] = Span(a.ctypes.data, a.size)
                outs[i] = Out(o.ctypes.data, o.size, 0)
            st = (ctypes.c_int * max(n, 1))()
            self._lib.gzgpu_decompress_batch(self._h, spans, n, outs, st)
            retry = [i for i in range(n) if st[i] == OUT_TOO_SMALL]
            if retry:
                caps = [outs[i].len if st[i] == OUT_TOO_SMALL else caps[i] for i in range(n)]
                continue
            res = []
            for i in range(n):
                if st[i] == OK:
                    res.append(outs_np[i][:outs[i].len].tobytes())
                elif st[i] == NOT_GZIP:
                    res.append(b"")
                else:
                    res.append(GzippyError("Decompression", strerror(st[i]), st[i]))
            return res
        raise GzippyError("Decompression", "output sizing failed")


def _ctx() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context()
    return _default_ctx


def decompress(data) -> bytes:
    """gzippy::decompress (src/lib.rs:176)."""
    return _ctx().decompress(data)


def decompress_with_threads(data, threads: int) -> bytes:
    """gzippy::decompress_with_threads (src/lib.rs:189)."""
    return _ctx().decompress(data)


def decompress_raw(data) -> bytes:
    """gzippy::decompress_raw (src/lib.rs:250): one raw DEFLATE stream."""
    return _ctx().inflate_raw(data)


deflate_decode = decompress_raw  # the reference's alias (src/lib.rs:258)


def decompress_zlib(data) -> bytes:
    """zlib data (decompress_zlib_turbo, src/decompress/mod.rs:895)."""
    return _ctx().inflate_zlib(data)


def build_index(data, interval_bytes: int = 1 << 20) -> bytes:
    """gzippy's seek index of a single-member gzip buffer (index.rs:55)."""
    return _ctx().build_index(data, interval_bytes)


def parse_index(blob: bytes):
    """(deflate offset, output size, [(bit offset, output offset, window)])
    of a version 1 index (load_index, src/decompress/index.rs:185-290)."""
    import struct
    if blob[:6] != b"GZIDX\x01":
        raise GzippyError("Parse", "not a version 1 seek index")
    doff, total, n, _ = struct.unpack_from("<IQIH", blob, 6)
    pts, at = [], 24
    for _ in range(n):
        b, o = struct.unpack_from("<QQ", blob, at)
        pts.append((b, o, blob[at + 16:at + 16 + 32768]))
        at += 16 + 32768
    return doff, total, pts


def decompress_to_writer(data, writer) -> int:
    """gzippy::decompress_to_writer (src/lib.rs:204)."""
    return _ctx().decompress_to_writer(data, writer)


def decompress_to_writer_with_threads(data, writer, threads: int) -> int:
    """gzippy::decompress_to_writer_with_threads (src/lib.rs:221)."""
    return _ctx().decompress_to_writer(data, writer)


def decompress_device_noalloc(d_in: int, in_len: int, d_out: int, out_cap: int,
                              cuda_stream: int = 0) -> int:
    """Decode without allocating device memory (include/gzgpu.h,
    gzgpu_decompress_device_noalloc): for callers that cannot call cudaMalloc,
    e.g. under a pool-only allocator or with all device memory reserved.  Raw
    device pointers on the current device; output limited to
    NOALLOC_MAX_OUT bytes.  Returns bytes written; raises GzippyError."""
    n = ctypes.c_size_t(0)
    rc = lib().gzgpu_decompress_device_noalloc(d_in, in_len, d_out, out_cap, ctypes.byref(n),
                                               cuda_stream or None)
    if rc == NOT_GZIP:
        return 0
    if rc != OK:
        if rc == OUT_TOO_SMALL:
            e = GzippyError("Decompression", f"output needs {n.value} bytes", rc)
            e.needed = n.value
            raise e
        _raise(rc)
    return n.value


class Server:
    """Continuous-batching decompression service (gzgpu_server_*, no reference
    counterpart).  submit() queues a gzip buffer and returns a ticket;
    result() / poll() give its bytes.  Requests run in lanes (contexts with
    their own CUDA streams) that overlap on the GPU, admitted against a
    device-memory budget; small requests share batches."""

    def __init__(self, device: int = 0, lanes: int = 4, budget_bytes: int = 0,
                 max_batch_bytes: int = 0, max_batch_requests: int = 0, large_bytes: int = 0,
                 autotune: bool = False, small_lanes: int = 0):
        self._lib = lib()
        cfg = ServerConfig(device, lanes, int(autotune), small_lanes, budget_bytes, max_batch_bytes,
                           max_batch_requests, large_bytes)
        h = ctypes.c_void_p()
        rc = self._lib.gzgpu_server_create(ctypes.byref(h), ctypes.byref(cfg))
        if rc != OK:
            _raise(rc)
        self._h = h
        self._keep = {}  # ticket -> (input, output) arrays held until done

    def close(self):
        if self._h:
            self._lib.gzgpu_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def submit(self, data, out_cap: int | None = None, out: np.ndarray | None = None) -> int:
        a = _as_u8(data)
        if out is None:
            if out_cap is None:
                isize = int(a[-4:].view("<u4")[0]) if a.size >= 4 else 0
                out_cap = max(isize, a.size * 4, 1 << 12)
            out = np.empty(out_cap, np.uint8)
        t = ctypes.c_uint64(0)
        rc = self._lib.gzgpu_submit(self._h, a.ctypes.data, a.size, out.ctypes.data, out.size,
                                    ctypes.byref(t))
        if rc != OK:
            _raise(rc)
        self._keep[t.value] = (a, out)
        return t.value

    def poll(self, ticket: int, wait_ms: int = -1, copy: bool = True):
        """(status, data or None, RequestTimes); status PENDING while running.
        A finished ticket is released.  data is bytes, or with copy=False a
        numpy view of the output buffer (no copy)."""
        n = ctypes.c_size_t(0)
        tm = RequestTimes()
        rc = self._lib.gzgpu_poll(self._h, ticket, wait_ms, ctypes.byref(n), ctypes.byref(tm))
        if rc == PENDING:
            return rc, None, tm
        _, out = self._keep.pop(ticket, (None, None))
        if rc in (OK, NOT_GZIP):
            if out is None:
                return rc, (b"" if copy else np.empty(0, np.uint8)), tm
            return rc, (out[:n.value].tobytes() if copy else out[:n.value]), tm
        return rc, None, tm

    def result(self, ticket: int, copy: bool = True):
        rc, data, _ = self.poll(ticket, -1, copy)
        if rc not in (OK, NOT_GZIP):
            _raise(rc)
        return data

    def stats(self) -> ServerStats:
        s = ServerStats()
        self._lib.gzgpu_server_get_stats(self._h, ctypes.byref(s))
        return s


def decompress_batch(datas) -> list:
    """Many independent streams in one job (no reference counterpart)."""
    return _ctx().decompress_batch(datas)
