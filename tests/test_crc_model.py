"""The CRC32 pass's arithmetic, restated on the CPU and checked against zlib.

The device pass (gzippy_b200/csrc/resolve.cu, crc_blocks_kernel and
member_check_kernel) never combines block CRCs in order.  It relies on four
facts about the reflected CRC-32 (polynomial 0xEDB88320), which this test
pins with the same block, slice and shift layout the kernel uses:
  * a register s followed by n zero bytes becomes A^n(s) = s * x^(8n) mod P;
  * raw(M1 | M2) = A^|M2|(raw(M1)) ^ raw(M2), raw() starting from 0 -- the
    same quantities gzippy combines in order (src/decompress/parallel/
    crc32.rs combine_crc32 :127);
  * leading zero bytes leave raw() at 0, so every lane slice can be given one
    length, counted back from its block's end;
  * crc(M) = ~(A^|M|(0xFFFFFFFF) ^ raw(M)).
Each block's raw CRC is moved to its member's end and XORed in, so blocks
fold in any order; the test shuffles them.
"""
import random
import zlib

import pytest

POLY = 0xEDB88320
BLOCK = 32768          # kCrcBlock
SLICE = BLOCK // 32    # kCrcSlice: one lane's bytes


def mulmod(a: int, b: int) -> int:
    """a * b mod P in the reflected representation (bit 31 = x^0)."""
    r = 0
    for i in range(31, -1, -1):
        if (a >> i) & 1:
            r ^= b
        b = (b >> 1) ^ (POLY if b & 1 else 0)
    return r


X2N = []
_v = 1 << 30  # x^1
for _ in range(64):
    X2N.append(_v)
    _v = mulmod(_v, _v)


def x_pow_8n(n: int) -> int:
    """x^(8n) mod P as a product over the bits of the exponent."""
    p, e, k = 1 << 31, n << 3, 0
    while e:
        if e & 1:
            p = mulmod(X2N[k], p)
        e >>= 1
        k += 1
    return p


TABLE = []
for _i in range(256):
    _c = _i
    for _ in range(8):
        _c = (_c >> 1) ^ (POLY if _c & 1 else 0)
    TABLE.append(_c)


def raw_crc(data: bytes) -> int:
    c = 0
    for b in data:
        c = TABLE[(c ^ b) & 0xFF] ^ (c >> 8)
    return c


# shift tables of the lane tree: level j moves a register past 2^j slices
SHIFT = [[[mulmod(x_pow_8n(SLICE << j), v << (8 * k)) for v in range(256)] for k in range(4)]
         for j in range(5)]


def shift(s: int, j: int) -> int:
    t = SHIFT[j]
    return t[0][s & 255] ^ t[1][(s >> 8) & 255] ^ t[2][(s >> 16) & 255] ^ t[3][s >> 24]


def block_raw(block: bytes) -> int:
    """One warp's work: 32 slices counted back from the block's end (bytes
    before the block are zeros), then a 5-level tree of fixed shifts."""
    n = len(block)
    regs = []
    for lane in range(32):
        end = n - SLICE * (31 - lane)
        start = max(0, end - SLICE)
        regs.append(raw_crc(block[start:end]) if end > 0 else 0)
    for j in range(5):
        d = 1 << j
        for lane in range(0, 32, 2 * d):
            regs[lane] = shift(regs[lane], j) ^ regs[lane + d]
    return regs[0]


def member_crc(member: bytes, seed: int) -> int:
    blocks = [(off, member[off:off + BLOCK]) for off in range(0, len(member), BLOCK)]
    random.Random(seed).shuffle(blocks)  # any order
    acc = 0
    for off, blk in blocks:
        after = len(member) - (off + len(blk))
        acc ^= mulmod(x_pow_8n(after), block_raw(blk))
    return ~(mulmod(x_pow_8n(len(member)), 0xFFFFFFFF) ^ acc) & 0xFFFFFFFF


@pytest.mark.parametrize("size", [0, 1, 1023, SLICE, BLOCK - 1, BLOCK, BLOCK + 1, 70001])
def test_block_crc_arithmetic_matches_zlib(size):
    data = bytes(random.Random(size).getrandbits(8) for _ in range(size))
    assert member_crc(data, seed=size) == zlib.crc32(data)


def test_shift_is_appending_zero_bytes():
    data = b"gzippy block"
    for n in (0, 1, 7, SLICE, 3 * BLOCK + 5):
        assert mulmod(x_pow_8n(n), raw_crc(data)) == raw_crc(data + bytes(n))
