"""Generate the golden gzip fixtures in this directory.

Each fixture is a small gzip input plus its expected result (status and the
SHA-256 and length of the decompressed bytes).  Expected outputs come from
construction (the plaintext the fixture was made from), cross-checked with
Python's zlib; the CUDA path and the oracle must both reproduce them.

Run:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys
import zlib

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from gzippy_b200 import workloads as W  # noqa: E402

OK, NOT_GZIP, BAD_HEADER, BAD_DEFLATE, CRC_MISMATCH, SIZE_MISMATCH = 0, 1, 2, 3, 4, 5
TRUNCATED = 9


def gz(data: bytes, level=6, strategy=zlib.Z_DEFAULT_STRATEGY) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, 31, 8, strategy)
    return c.compress(data) + c.flush()


def gz_sync(data: bytes, piece: int) -> bytes:
    """one member whose body has Z_SYNC_FLUSH points (empty stored blocks)"""
    c = zlib.compressobj(6, zlib.DEFLATED, 31)
    out = b""
    for i in range(0, len(data), piece):
        out += c.compress(data[i:i + piece]) + c.flush(zlib.Z_SYNC_FLUSH)
    return out + c.flush()


def header_member(data: bytes) -> bytes:
    raw = zlib.compressobj(6, zlib.DEFLATED, -15)
    body = raw.compress(data) + raw.flush()
    h = bytes([0x1f, 0x8b, 8, 0x1e, 1, 2, 3, 4, 0, 3])          # FHCRC|FEXTRA|FNAME|FCOMMENT
    h += (7).to_bytes(2, "little") + b"ab\x03\x00xyz"
    h += b"fixture.bin\x00" + b"golden fixture\x00"
    h += (zlib.crc32(h) & 0xFFFF).to_bytes(2, "little")
    return h + body + zlib.crc32(data).to_bytes(4, "little") + (len(data) & 0xFFFFFFFF).to_bytes(4, "little")


def main():
    text = W.content(W.MARKOV, 77, 1 << 20).tobytes()
    rnd = W.content(W.RANDOM, 78, 64 << 10).tobytes()
    runs = W.content(W.RUNS, 79, 300 << 10).tobytes()
    ramps = W.content(W.RAMPS, 80, 120 << 10).tobytes()
    small = text[:100_000]
    cases = []

    def add(name, blob, expected, status=OK):
        cases.append((name, blob, expected, status))

    add("empty_member", gz(b""), b"")
    add("one_byte", gz(b"x", 9), b"x")
    add("text_1m_l9", gz(text, 9), text)
    add("text_100k_l6", gz(small, 6), small)
    add("random_stored", gz(rnd, 6), rnd)
    add("runs_l9", gz(runs, 9), runs)
    add("ramps_fixed_l1", gz(ramps, 1, zlib.Z_FIXED), ramps)
    add("text_fixed_l1", gz(small, 1, zlib.Z_FIXED), small)
    add("level0_stored", gz(ramps[:70000], 0), ramps[:70000])
    add("sync_flush", gz_sync(small, 7000), small)
    parts = [small[:30000], rnd[:20000], runs[:50000], b"", ramps[:40000]]
    add("multi_member", b"".join(gz(p, l) for p, l in zip(parts, [6, 9, 1, 6, 6])), b"".join(parts))
    add("header_fields", header_member(small), small)
    add("trailing_garbage", gz(small) + b"\x00garbage after the member\xff", small)
    add("two_empty_members", gz(b"") + gz(b""), b"")
    add("not_gzip", b"plain text, not gzip", b"", NOT_GZIP)
    add("empty_input", b"", b"", NOT_GZIP)
    add("magic_only", b"\x1f\x8b", b"", TRUNCATED)
    good = gz(small)
    add("truncated_body", good[: len(good) // 2], b"", TRUNCATED)
    add("truncated_trailer", good[:-3], b"", TRUNCATED)
    bad = bytearray(good)
    bad[-8] ^= 0x01
    add("crc_mismatch", bytes(bad), b"", CRC_MISMATCH)
    bad = bytearray(good)
    bad[-1] ^= 0x10
    add("isize_mismatch", bytes(bad), b"", SIZE_MISMATCH)
    bad = bytearray(good)
    bad[3] = 0xE0
    add("reserved_flags", bytes(bad), b"", BAD_HEADER)
    bad = bytearray(good)
    bad[2] = 7
    add("bad_method", bytes(bad), b"", BAD_HEADER)
    bad = bytearray(good)
    bad[10] = 0xFF          # first block header: BTYPE=11 (reserved)
    add("reserved_btype", bytes(bad), b"", BAD_DEFLATE)

    manifest = []
    for name, blob, expected, status in cases:
        if status == OK:
            # independent check of the expected output with zlib (multi-member aware)
            d = zlib.decompressobj(31)
            got, rest = b"", blob
            while rest:
                d = zlib.decompressobj(31)
                got += d.decompress(rest)
                rest = d.unused_data
                if not rest.startswith(b"\x1f\x8b"):
                    break
            assert got == expected, name
        path = os.path.join(HERE, name + ".gz")
        with open(path, "wb") as f:
            f.write(blob)
        manifest.append({"name": name, "file": name + ".gz", "status": status,
                         "out_len": len(expected), "sha256": hashlib.sha256(expected).hexdigest()})
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(f"{len(manifest)} fixtures, {sum(len(c[1]) for c in cases)} bytes")


if __name__ == "__main__":
    main()
