"""gzippy's "GZ" multi-block format and BGZF (parse_bgzf_blocks,
src/decompress/bgzf.rs:43-160; detection has_bgzf_markers,
src/decompress/format.rs:13): every block is a complete gzip member whose
FEXTRA carries its size, in a "GZ" subfield (4-byte size, or the legacy
2-byte size - 1) or a BGZF "BC" subfield (size - 1), ending with BGZF's
empty EOF block.  The device decodes such files through its member-parallel
path (members found by the device scan, each decoded independently, CRC32
and ISIZE checked per member); results are byte-exact against the oracle
and zlib."""
import struct
import zlib

import pytest

from gzippy_b200 import workloads as W
from oracle import pyoracle as O


def _deflate(p: bytes, level: int) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, -15)
    return c.compress(p) + c.flush()


def block(p: bytes, level: int, form: str) -> bytes:
    """One member of the multi-block format; form in {"gz4", "gz2", "bc"}."""
    d = _deflate(p, level)
    trailer = struct.pack("<II", zlib.crc32(p), len(p) & 0xFFFFFFFF)
    if form == "gz4":
        total = 10 + 2 + 8 + len(d) + 8
        extra = b"GZ" + struct.pack("<HI", 4, total)
    else:
        total = 10 + 2 + 6 + len(d) + 8
        extra = (b"GZ" if form == "gz2" else b"BC") + struct.pack("<HH", 2, total - 1)
    hdr = b"\x1f\x8b\x08\x04" + b"\x00\x00\x00\x00" + b"\x00\xff" + struct.pack("<H", len(extra))
    m = hdr + extra + d + trailer
    assert len(m) == total
    return m


BGZF_EOF = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")


def multiblock(form: str, total: int, block_bytes: int, seed: int):
    plain = b"".join(W.content(k % 4, seed + k, block_bytes).tobytes()
                     for k in range((total + block_bytes - 1) // block_bytes))[:total]
    blocks = [block(plain[i:i + block_bytes], (1, 6, 9)[(i // block_bytes) % 3], form)
              for i in range(0, len(plain), block_bytes)]
    data = b"".join(blocks) + (BGZF_EOF if form == "bc" else b"")
    return plain, data


FORMS = [("gz4", 1 << 20), ("gz2", 60 << 10), ("bc", 60 << 10)]


def test_eof_block_is_an_empty_member():
    assert zlib.decompress(BGZF_EOF, 31) == b""


@pytest.mark.parametrize("form,bb", FORMS)
def test_oracle_multiblock(form, bb):
    plain, data = multiblock(form, 3 << 20, bb, 800)
    st, out = O.decompress(data, cap=len(plain) + 4096)
    assert st == 0 and out.tobytes() == plain


@pytest.mark.gpu
@pytest.mark.parametrize("form,bb", FORMS)
def test_device_multiblock(form, bb):
    import gzippy_b200 as G
    plain, data = multiblock(form, 40 << 20, bb, 810)
    cx = G.Context()
    try:
        assert cx.decompress(data) == plain
        # a corrupt CRC in one block fails the whole file
        bad = bytearray(data)
        first = block(plain[:bb], 1, form)
        bad[len(first) - 8] ^= 1
        with pytest.raises(G.GzippyError):
            cx.decompress(bytes(bad))
    finally:
        cx.close()
