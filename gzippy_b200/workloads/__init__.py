"""Seeded synthetic gzip workloads (the five decompression configurations).

Every workload is generated on the machine that runs it from a seed, so no
data files travel.  Content types and the zlib encoder stand-in are
described in ``synth.c``.  Every member is one serial zlib deflate stream
(``encoder="zlib-serial"``); the pigz-style framing (parallel pieces closed
by Z_SYNC_FLUSH, which leaves an empty stored block every piece) is only
used when a caller names it (``encoder="pigz"``).

Configurations (sizes scale with ``scale`` for tests):

* ``single_member_text``   -- 64 MiB Markov text, level 6, one member.
* ``single_member_mixed``  -- 256 x 4 MiB segments cycling the four content
  types (1 GiB), level 6, one member.
* ``multi_member``         -- 2048 members x 2 MiB, type and level in {1,6,9}
  drawn per member, concatenated.
* ``stream_batch``         -- 10,000 independent streams, log-normal sizes
  (median 64 KiB, sigma 1.5, clamped 1 KiB..64 MiB).
* ``serving_requests``     -- Poisson arrivals, sizes log-uniform 4-256 KiB
  (p=0.8) or 8-512 MiB (p=0.2).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsynth.so")
SRC = os.path.join(HERE, "synth.c")

MARKOV, RANDOM, RUNS, RAMPS = 0, 1, 2, 3
SEG = 4 << 20
_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", LIB, SRC,
                               "-lz", "-lm", "-lpthread"])
    return LIB


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(LIB)
            L.syn_content.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t]
            L.syn_gzip.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_size_t]
            L.syn_gzip.restype = ctypes.c_size_t
            L.syn_gzip_parallel.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p,
                                            ctypes.c_size_t]
            L.syn_gzip_parallel.restype = ctypes.c_size_t
            L.syn_gzip_bound.argtypes = [ctypes.c_size_t]
            L.syn_gzip_bound.restype = ctypes.c_size_t
            _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def content(ctype: int, seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint8)
    if n:
        lib().syn_content(int(ctype), int(seed) & (2**64 - 1), _ptr(out), n)
    return out


def gzip_member(plain: np.ndarray, level: int, threads: int = 1,
                block: int = 1 << 20) -> np.ndarray:
    """One gzip member of `plain` (pigz-style parallel when threads > 1)."""
    plain = np.ascontiguousarray(plain, dtype=np.uint8)
    n = plain.size
    cap = lib().syn_gzip_bound(n)
    out = np.empty(cap, dtype=np.uint8)
    if threads > 1 and n > block:
        k = lib().syn_gzip_parallel(_ptr(plain), n, level, threads, block, _ptr(out), cap)
    else:
        k = lib().syn_gzip(_ptr(plain), n, level, _ptr(out), cap)
    if k == 0:
        raise RuntimeError("zlib compression failed")
    return out[:k].copy()


def _cpus() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:  # pragma: no cover
        return os.cpu_count() or 1


@dataclass
class Workload:
    name: str
    compressed: list            # list of np.uint8 arrays (one per stream)
    plain_sizes: list           # uncompressed size per stream
    plain: list = field(default_factory=list)   # kept only when asked
    meta: dict = field(default_factory=dict)

    @property
    def total_in(self) -> int:
        return int(sum(c.size for c in self.compressed))

    @property
    def total_out(self) -> int:
        return int(sum(self.plain_sizes))


ENCODERS = ("zlib-serial", "pigz")


def encode_member(plain: np.ndarray, level: int, encoder: str = "zlib-serial",
                  threads: int | None = None) -> np.ndarray:
    """One gzip member: one serial deflate stream ("zlib-serial"), or the
    pigz-style framing of 1 MiB pieces on `threads` threads ("pigz")."""
    if encoder == "zlib-serial":
        return gzip_member(plain, level, 1)
    if encoder == "pigz":
        return gzip_member(plain, level, threads or _cpus())
    raise ValueError(f"unknown encoder {encoder!r}")


def single_member_text(seed: int = 1234, size: int = 64 << 20, level: int = 6,
                       keep_plain: bool = False, threads: int | None = None,
                       encoder: str = "zlib-serial") -> Workload:
    plain = content(MARKOV, seed, size)
    comp = encode_member(plain, level, encoder, threads)
    return Workload("single_member_text", [comp], [size], [plain] if keep_plain else [],
                    {"level": level, "seed": seed, "encoder": encoder})


def single_member_mixed(seed: int = 1235, segments: int = 256, seg_bytes: int = SEG,
                        level: int = 6, keep_plain: bool = False,
                        threads: int | None = None, encoder: str = "zlib-serial") -> Workload:
    plain = np.empty(segments * seg_bytes, dtype=np.uint8)
    th = threads or _cpus()

    def one(i):
        plain[i * seg_bytes:(i + 1) * seg_bytes] = content(i % 4, seed * 1000003 + i, seg_bytes)

    with ThreadPoolExecutor(th) as ex:
        list(ex.map(one, range(segments)))
    comp = encode_member(plain, level, encoder, th)
    return Workload("single_member_mixed", [comp], [plain.size], [plain] if keep_plain else [],
                    {"level": level, "seed": seed, "segments": segments, "seg_bytes": seg_bytes,
                     "encoder": encoder})


def multi_member(seed: int = 1236, members: int = 2048, member_bytes: int = 2 << 20,
                 keep_plain: bool = False, threads: int | None = None) -> Workload:
    rng = np.random.default_rng(seed)
    types = rng.integers(0, 4, members)
    levels = rng.choice([1, 6, 9], members)
    parts = [None] * members
    plains = [None] * members

    def one(i):
        p = content(int(types[i]), seed * 7919 + i, member_bytes)
        parts[i] = gzip_member(p, int(levels[i]))
        if keep_plain:
            plains[i] = p

    with ThreadPoolExecutor(threads or _cpus()) as ex:
        list(ex.map(one, range(members)))
    comp = np.concatenate(parts)
    plain = [np.concatenate(plains)] if keep_plain else []
    return Workload("multi_member", [comp], [members * member_bytes], plain,
                    {"members": members, "member_bytes": member_bytes,
                     "types": types.tolist(), "levels": levels.tolist(),
                     "member_comp_bytes": [int(x.size) for x in parts]})


def lognormal_sizes(rng, n, median=64 << 10, sigma=1.5, lo=1 << 10, hi=64 << 20):
    s = np.exp(rng.normal(np.log(median), sigma, n))
    return np.clip(s, lo, hi).astype(np.int64)


def stream_batch(seed: int = 1237, streams: int = 10000, keep_plain: bool = False,
                 threads: int | None = None, max_size: int = 64 << 20) -> Workload:
    rng = np.random.default_rng(seed)
    sizes = lognormal_sizes(rng, streams, hi=max_size)
    types = rng.integers(0, 4, streams)
    levels = rng.choice([1, 6, 9], streams)
    comps = [None] * streams
    plains = [None] * streams

    def one(i):
        p = content(int(types[i]), seed * 104729 + i, int(sizes[i]))
        comps[i] = gzip_member(p, int(levels[i]))
        if keep_plain:
            plains[i] = p

    with ThreadPoolExecutor(threads or _cpus()) as ex:
        list(ex.map(one, range(streams)))
    return Workload("stream_batch", comps, sizes.tolist(), plains if keep_plain else [],
                    {"types": types.tolist(), "levels": levels.tolist()})


def serving_requests(seed: int = 1238, rate_hz: float = 20.0, duration_s: float = 60.0,
                     small=(4 << 10, 256 << 10), large=(8 << 20, 512 << 20), p_small=0.8):
    """Arrival times and request specs (size, type, level) for the serving loop."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            break
        lo, hi = small if rng.random() < p_small else large
        size = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        out.append((t, size, int(rng.integers(0, 4)), int(rng.choice([1, 6, 9]))))
    return out


def serving_pool(seed: int = 1238, n: int = 64, small=(4 << 10, 256 << 10),
                 large=(8 << 20, 512 << 20), p_small=0.8, threads: int | None = None):
    """n distinct serving requests: uncompressed size log-uniform in `small`
    with probability p_small, else log-uniform in `large`; content type
    uniform over the four kinds, level uniform in {1, 6, 9}.  Returns
    (compressed arrays, plain sizes, plain CRC32s, specs)."""
    import zlib
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        lo, hi = small if rng.random() < p_small else large
        size = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        specs.append((size, int(rng.integers(0, 4)), int(rng.choice([1, 6, 9]))))
    comps, crcs = [None] * n, [0] * n

    def one(i):
        size, ctype, level = specs[i]
        p = content(ctype, seed * 7907 + i, size)
        comps[i] = gzip_member(p, level)
        crcs[i] = zlib.crc32(p)

    with ThreadPoolExecutor(threads or _cpus()) as ex:
        list(ex.map(one, range(n)))
    return comps, [s[0] for s in specs], crcs, specs


def poisson_arrivals(seed: int, rate_hz: float, duration_s: float, n_pool: int):
    """Arrival times of a Poisson process over duration_s, each with a pool index."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            return out
        out.append((t, int(rng.integers(0, n_pool))))

