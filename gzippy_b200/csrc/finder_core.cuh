// finder_core.cuh -- block-start predicate and warp search, shared by the
// finder kernel and the inflate kernel's next-candidate retry.
//
// Predicate of the reference (src/decompress/parallel/blockfinder_validation.rs):
//   dynamic: BFINAL=0, BTYPE=10, HLIT<=29, HDIST<=29 (13-bit filter,
//            :68-150); precode leaf count 128 or 64 (validate_precode
//            :190-226) and Kraft-exact (is_valid_huffman_lengths :807-830);
//            the HLIT+257+HDIST+1 code lengths decode with the precode,
//            EOB has a code, litlen and dist sets are Kraft-exact
//            (validate_huffman_codes :836-925).  No fixed-Huffman candidates.
//   stored:  LEN == ~NLEN at a byte boundary preceded by 3 zero header bits;
//            the candidate spans [byte_bit - zero_run, byte_bit - 3]
//            (find_uncompressed_blocks :370-475).
#pragma once
#include <cstdint>

#include "common.cuh"

namespace gzgpu {

static __constant__ uint8_t f_cl_order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// bits [bit, bit+k) of the input, k <= 57; bits at or past the stream end
// (byte `nbytes`) read 0.  Three aligned 32-bit loads (the buffer is padded).
static __device__ __forceinline__ uint64_t peek_bits(const uint8_t* in, uint64_t nbytes, uint64_t bit,
                                                     int k) {
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  const uint64_t wi = bit >> 5;
  const int sh = (int)(bit & 31);
  const uint64_t a = ((uint64_t)in32[wi + 1] << 32) | in32[wi];
  uint64_t v = (a >> sh) | (sh ? (uint64_t)in32[wi + 2] << (64 - sh) : 0);
  uint64_t avail = nbytes * 8 > bit ? nbytes * 8 - bit : 0;
  int kk = avail < (uint64_t)k ? (int)avail : k;
  return kk ? v & (~0ull >> (64 - kk)) : 0;
}

// Kraft equality over 15-bit leaves, or a single one-bit code.
static __device__ __forceinline__ bool kraft_exact(uint32_t leaves, uint32_t gt1) {
  if (leaves == (1u << 14)) return gt1 == 0;
  return leaves == (1u << 15);
}

// Bits [bit, bit + 96) of the stream as (lo64, hi32), from four aligned
// 32-bit loads; bits at or past the stream end read 0 (the buffer is padded,
// so the loads stay inside it).
static __device__ __forceinline__ void load_bits96(const uint8_t* in, uint64_t nbytes,
                                                   uint64_t bit, uint64_t& x, uint32_t& xh) {
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  const uint64_t wi = bit >> 5;
  const uint32_t w0 = in32[wi], w1 = in32[wi + 1], w2 = in32[wi + 2], w3 = in32[wi + 3];
  const int sh = (int)(bit & 31);
  const uint64_t a = ((uint64_t)w1 << 32) | w0, b = ((uint64_t)w3 << 32) | w2;
  x = sh ? (a >> sh) | (b << (64 - sh)) : a;
  xh = (uint32_t)(b >> sh);
  const uint64_t nbits = nbytes * 8;
  if (bit + 96 > nbits) {
    const uint64_t valid = nbits > bit ? nbits - bit : 0;
    if (valid < 64) {
      x &= valid ? (~0ull >> (64 - valid)) : 0;
      xh = 0;
    } else {
      xh &= valid > 64 ? (0xFFFFFFFFu >> (96 - valid)) : 0;
    }
  }
}

// Leaf count of 4 precode lengths (3 bits each) packed in 12 bits: the
// table of validate_precode (blockfinder_validation.rs:148-226).
static __device__ __forceinline__ uint32_t precode_leaves4(uint32_t v) {
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    uint32_t L = (v >> (3 * i)) & 7;
    s += L ? 1u << (7 - L) : 0u;
  }
  return s;
}

// Rest of the dynamic-header predicate once the 13-bit filter and the
// precode leaf count have passed: Kraft-exact precode, code lengths decode,
// EOB present, Kraft-exact litlen and dist sets.
static __device__ __noinline__ bool dyn_candidate_full(const uint8_t* in, uint64_t nbytes,
                                                       uint64_t bit) {
  const uint64_t nbits = nbytes * 8;
  uint32_t h = (uint32_t)peek_bits(in, nbytes, bit, 17);
  int hlit = (h >> 3) & 31, hdist = (h >> 8) & 31, pc = ((h >> 13) & 15) + 4;
  uint64_t pbits = peek_bits(in, nbytes, bit + 17, 3 * pc);
  uint32_t leaves15 = 0, gt1 = 0;
  uint8_t cl[19];
#pragma unroll
  for (int i = 0; i < 19; i++) cl[i] = 0;
  for (int i = 0; i < pc; i++) {
    uint32_t L = (uint32_t)(pbits >> (3 * i)) & 7;
    cl[f_cl_order[i]] = (uint8_t)L;
    if (L) {
      leaves15 += 1u << (15 - L);
      gt1 += L > 1;
    }
  }
  if (!kraft_exact(leaves15, gt1)) return false;
  // canonical precode tables
  uint16_t cnt[8], first[8], offs[8];
  uint8_t sorted[19];
#pragma unroll
  for (int L = 0; L < 8; L++) cnt[L] = 0;
  for (int s = 0; s < 19; s++) cnt[cl[s]]++;
  cnt[0] = 0;
  {
    uint32_t code = 0, off = 0;
    for (int L = 1; L < 8; L++) {
      if (L > 1) code = (code + cnt[L - 1]) << 1;
      first[L] = (uint16_t)code;
      offs[L] = (uint16_t)off;
      off += cnt[L];
    }
    uint16_t nx[8];
    for (int L = 0; L < 8; L++) nx[L] = offs[L];
    for (int s = 0; s < 19; s++)
      if (cl[s]) sorted[nx[cl[s]]++] = (uint8_t)s;
  }
  // decode the litlen + dist code lengths, accumulating Kraft sums
  const int hl = 257 + hlit, total = hl + 1 + hdist;
  uint64_t pos = bit + 17 + 3 * pc;
  uint32_t lit_leaves = 0, lit_gt1 = 0, dist_leaves = 0, dist_gt1 = 0;
  int i = 0;
  uint32_t prev = 0, eob_len = 0;
  while (i < total) {
    if (pos >= nbits) return false;
    uint32_t w = (uint32_t)peek_bits(in, nbytes, pos, 14);
    // MSB-first 7-bit code
    uint32_t rev = __brev(w) >> 25;
    int sym = -1;
    for (int L = 1; L < 8; L++) {
      uint32_t c = rev >> (7 - L);
      uint32_t idx = c - first[L];
      if (idx < cnt[L]) {
        sym = sorted[offs[L] + idx];
        pos += L;
        break;
      }
    }
    if (sym < 0) return false;
    uint32_t v;
    int rep;
    if (sym < 16) {
      v = sym;
      rep = 1;
    } else if (sym == 16) {
      if (i == 0) return false;
      v = prev;
      rep = 3 + (int)peek_bits(in, nbytes, pos, 2);
      pos += 2;
    } else if (sym == 17) {
      v = 0;
      rep = 3 + (int)peek_bits(in, nbytes, pos, 3);
      pos += 3;
    } else {
      v = 0;
      rep = 11 + (int)peek_bits(in, nbytes, pos, 7);
      pos += 7;
    }
    if (i + rep > total) return false;
    if (pos > nbits) return false;
    if (v) {
      int n_lit = i < hl ? min(rep, hl - i) : 0;
      int n_dist = rep - n_lit;
      lit_leaves += (uint32_t)n_lit << (15 - v);
      dist_leaves += (uint32_t)n_dist << (15 - v);
      if (v > 1) {
        lit_gt1 += n_lit;
        dist_gt1 += n_dist;
      }
      if (i <= 256 && 256 < i + rep) eob_len = v;
      // Kraft sums only grow: an over-subscribed set fails the final test
      if (lit_leaves > (1u << 15) || dist_leaves > (1u << 15)) return false;
    }
    prev = v;
    i += rep;
  }
  if (eob_len == 0) return false;
  return kraft_exact(lit_leaves, lit_gt1) && kraft_exact(dist_leaves, dist_gt1);
}

// The cheap part of the dynamic-header predicate at `bit`: the 13-bit header
// filter and the precode leaf count via `leaf_lut` (the 4096-entry leaf-count
// table, or null to count arithmetically).  dyn_candidate_fast adds
// dyn_candidate_full.
static __device__ __forceinline__ bool dyn_leaf_ok(const uint8_t* in, uint64_t nbytes, uint64_t bit,
                                                   const uint16_t* leaf_lut) {
  if (bit + 17 > nbytes * 8) return false;
  uint64_t x;
  uint32_t xh;
  load_bits96(in, nbytes, bit, x, xh);
  const uint32_t h = (uint32_t)x;
  if ((h & 1) || ((h >> 1) & 3) != 2 || ((h >> 3) & 31) > 29 || ((h >> 8) & 31) > 29) return false;
  const int pc = ((h >> 13) & 15) + 4;
  if (bit + 17 + 3 * pc > nbytes * 8) return false;
  // precode bits [17, 17 + 3*pc) of the 96-bit window
  uint64_t pb = (x >> 17) | ((uint64_t)xh << 47);
  pb &= (1ull << (3 * pc)) - 1;
  uint32_t leaves;
  if (leaf_lut) {
    leaves = leaf_lut[pb & 0xFFF] + leaf_lut[(pb >> 12) & 0xFFF] + leaf_lut[(pb >> 24) & 0xFFF] +
             leaf_lut[(pb >> 36) & 0xFFF] + leaf_lut[pb >> 48];
  } else {
    leaves = precode_leaves4((uint32_t)(pb & 0xFFF)) + precode_leaves4((uint32_t)((pb >> 12) & 0xFFF)) +
             precode_leaves4((uint32_t)((pb >> 24) & 0xFFF)) +
             precode_leaves4((uint32_t)((pb >> 36) & 0xFFF)) + precode_leaves4((uint32_t)(pb >> 48));
  }
  return leaves == 128 || leaves == 64;
}

static __device__ __forceinline__ bool dyn_candidate_fast(const uint8_t* in, uint64_t nbytes,
                                                          uint64_t bit,
                                                          const uint16_t* leaf_lut) {
  return dyn_leaf_ok(in, nbytes, bit, leaf_lut) && dyn_candidate_full(in, nbytes, bit);
}

// The block after a true non-final stored block starts at byte `n` (its
// header's first bit is bit 0 of that byte): another stored block (LEN ==
// ~NLEN one byte on) or a dynamic block whose header passes the full
// predicate.  Not a rule of the reference's finder: it drops the false
// LEN/NLEN matches (about one per 64 KiB of random bytes) that would
// otherwise start speculative chunks inside stored data.  A true stored
// block followed by a fixed-Huffman block is given up as a start.
static __device__ __forceinline__ bool stored_successor_ok(const uint8_t* in, uint64_t nbytes,
                                                           uint64_t n) {
  if (n >= nbytes) return false;
  const uint32_t bt = (in[n] >> 1) & 3;
  if (bt == 0) {
    if (n + 5 > nbytes) return false;
    const uint32_t sz = in[n + 1] | (in[n + 2] << 8) | ((uint32_t)in[n + 3] << 16) |
                        ((uint32_t)in[n + 4] << 24);
    return ((sz ^ (sz >> 16)) & 0xFFFF) == 0xFFFF;
  }
  if (bt != 2) return false;
  const uint64_t bit = n * 8;
  if (bit + 17 > nbytes * 8) return false;
  const uint32_t h = (uint32_t)peek_bits(in, nbytes, bit, 13);
  if (((h >> 3) & 31) > 29 || ((h >> 8) & 31) > 29) return false;
  return dyn_candidate_full(in, nbytes, bit);
}

// A candidate found at seek bit `hi` stays a chunk start unless it is a stored
// block whose successor fails stored_successor_ok (the finder kernel then
// searches on from its first bit + 1; the decoder's in-kernel retry takes
// the reference's candidates as they are).
static __device__ __forceinline__ bool start_ok(const uint8_t* in, uint64_t nbytes, uint64_t hi) {
  if (((peek_bits(in, nbytes, hi, 3) >> 1) & 3) != 0) return true;
  const uint64_t off = (hi + 3) >> 3;
  const uint32_t len = in[off] | (in[off + 1] << 8);
  return stored_successor_ok(in, nbytes, off + 4 + len);
}

// Stored candidate test at byte offset `off` (find_uncompressed_blocks):
// LEN == ~NLEN at the byte boundary, 3 zero header bits before it; the
// candidate spans [byte_bit - zero_run, byte_bit - 3].
static __device__ __forceinline__ bool stored_candidate(const uint8_t* in, uint64_t nbytes,
                                                        uint64_t off, uint64_t from, uint64_t to,
                                                        uint64_t hi_to, uint64_t& lo, uint64_t& hi) {
  uint32_t sz = in[off] | (in[off + 1] << 8) | ((uint32_t)in[off + 2] << 16) |
                ((uint32_t)in[off + 3] << 24);
  if (((sz ^ (sz >> 16)) & 0xFFFF) != 0xFFFF) return false;
  uint64_t byte_bit = off * 8;
  uint32_t pre = (uint32_t)peek_bits(in, nbytes, byte_bit - 10, 10);
  if (pre & (7u << 7)) return false;
  int tz = 3;
  for (int j = 4; j <= 10; j++) {
    if (pre & (1u << (10 - j))) break;
    tz = j;
  }
  lo = byte_bit - tz;
  hi = byte_bit - 3;
  uint32_t len = sz & 0xFFFF;
  return lo >= from && lo < to && hi < hi_to && len != 0 && off + 4 + len <= nbytes;
}

// Bits [p, p + 64) of the stream from three aligned 32-bit loads (the buffer
// is padded past the stream; bits past its end are not masked here).
static __device__ __forceinline__ uint64_t bits64_at(const uint32_t* in32, uint64_t p) {
  const uint64_t wi = p >> 5;
  const int sh = (int)(p & 31);
  const uint64_t a = ((uint64_t)in32[wi + 1] << 32) | in32[wi];
  return sh ? (a >> sh) | ((uint64_t)in32[wi + 2] << (64 - sh)) : a;
}

// Positions i < 32 (bit i of the result) where the 13-bit dynamic header
// filter passes, for the 64 stream bits X starting at the first of them:
// BFINAL = 0, BTYPE = 10, HLIT <= 29 (not bits 4..7 all set), HDIST <= 29
// (not bits 9..12 all set).  All 32 positions at once, bit-parallel.
static __device__ __forceinline__ uint32_t dyn_filter32(uint64_t X) {
  const uint64_t hlit_big = (X >> 4) & (X >> 5) & (X >> 6) & (X >> 7);
  const uint64_t hdist_big = (X >> 9) & (X >> 10) & (X >> 11) & (X >> 12);
  return (uint32_t)(~X & ~(X >> 1) & (X >> 2) & ~hlit_big & ~hdist_big);
}

// Byte offsets k < 4 (bit k) among off .. off + 3 where LEN == ~NLEN, from
// the 7 bytes at off held in the low bits of B (bytes beyond are ignored).
static __device__ __forceinline__ uint32_t stored_filter4(uint64_t B) {
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t sz = (uint32_t)(B >> (8 * k));
    m |= (((sz ^ (sz >> 16)) & 0xFFFFu) == 0xFFFFu ? 1u : 0u) << k;
  }
  return m;
}

// First candidate in (bit_offset, seek_bit) order with bit_offset in
// [from, to) of the stream ending at byte `nbytes` (a stored candidate's
// seek bit must also be below hi_to); all 32 lanes call it together and get
// the same answer.  The range is walked in 1024-bit windows.  In each, every
// lane first screens 4 byte offsets for a stored block's LEN/NLEN pair, then
// 32 bit offsets with the 13-bit dynamic header filter, both bit-parallel,
// and runs the full tests only on the offsets that pass (about 1 in 9 bits);
// a ballot picks the lowest hit.  The first stored hit in byte order is the
// smallest stored candidate, so the dynamic scan only needs to reach it.
// Per-warp candidate lists of the grouped scan (finder kernel): positions of
// one 1024-bit window that pass the 13-bit filter, then positions of a group
// of windows that also pass the precode leaf count.
constexpr uint32_t kFindGroup = 4;    // 1024-bit windows screened before the full tests
constexpr uint32_t kFindFull = 64;    // leaf-count survivors held per group
struct FinderLists {
  uint16_t c1[1024];
  uint32_t c2[kFindFull];
  uint32_t n2;
};

static __device__ bool warp_find_first(const uint8_t* __restrict__ in, uint64_t nbytes,
                                       uint64_t from, uint64_t to, uint64_t hi_to, int lane,
                                       uint64_t& out_lo, uint64_t& out_hi,
                                       const uint16_t* leaf_lut = nullptr,
                                       FinderLists* L = nullptr, bool dyn_only = false);

// The same search with the dynamic tests spread over the warp: a group of
// kFindGroup windows is screened (13-bit filter per lane, then the leaf
// count for every survivor, 32 at a time), and the full tests of the group's
// survivors run one per lane, the lowest passing position winning.  Used by
// the finder kernel, whose warps have the lists in shared memory.  With
// `dyn_only` the stored candidates are not searched (the finder kernel runs
// after the stored-start pass, which took every stored candidate that could
// start its range).
static __device__ bool warp_find_first_grouped(const uint8_t* __restrict__ in, uint64_t nbytes,
                                               uint64_t from, uint64_t to, uint64_t hi_to,
                                               int lane, uint64_t& out_lo, uint64_t& out_hi,
                                               const uint16_t* leaf_lut, FinderLists* L,
                                               bool dyn_only) {
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  if (to > nbytes * 8) to = nbytes * 8;
  if (hi_to > nbytes * 8) hi_to = nbytes * 8;
  bool have = false;
  uint64_t best_lo = 0, best_hi = 0;
  const uint64_t until = nbytes >= 5 ? min((hi_to + 7) / 8, nbytes - 4) : 0;
  uint64_t next_off = max((from + 3 + 7) / 8, (uint64_t)2);
  for (uint64_t g0 = from; g0 < to; g0 += 1024 * kFindGroup) {
    const uint64_t g1 = min(g0 + 1024 * kFindGroup, to);
    const uint64_t off_end = min(until, (g1 + 10) / 8 + 1);
    while (!dyn_only && !have && next_off < off_end) {
      const uint64_t ob = next_off + 4 * (uint64_t)lane;
      uint32_t m = 0;
      if (ob < off_end) {
        m = stored_filter4(bits64_at(in32, ob * 8));
        if (ob + 4 > off_end) m &= (1u << (off_end - ob)) - 1;
      }
      uint64_t lo = 0, hi = 0;
      bool hit = false;
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        if (stored_candidate(in, nbytes, ob + k, from, to, hi_to, lo, hi)) {
          hit = true;
          break;
        }
      }
      const uint32_t b = __ballot_sync(0xFFFFFFFFu, hit);
      if (b) {
        const int src = __ffs(b) - 1;
        best_lo = __shfl_sync(0xFFFFFFFFu, lo, src);
        best_hi = __shfl_sync(0xFFFFFFFFu, hi, src);
        have = true;
      }
      next_off = min(next_off + 128, off_end);
    }
    const uint64_t lim = have ? min(g1, best_lo + 1) : g1;
    if (lane == 0) L->n2 = 0;
    __syncwarp();
    for (uint64_t w0 = g0; w0 < lim; w0 += 1024) {
      const uint64_t pl = w0 + 32 * (uint64_t)lane;
      uint32_t m = 0;
      if (pl < lim) {
        m = dyn_filter32(bits64_at(in32, pl));
        if (pl + 32 > lim) m &= (1u << (lim - pl)) - 1;
      }
      const uint32_t c = __popc(m);
      uint32_t incl = c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += v;
      }
      const uint32_t tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
      uint32_t k = incl - c;
      while (m) {
        const int i = __ffs(m) - 1;
        m &= m - 1;
        L->c1[k++] = (uint16_t)(32 * lane + i);
      }
      __syncwarp();
      for (uint32_t j = lane; j < tot; j += 32) {
        const uint64_t p = w0 + L->c1[j];
        if (dyn_leaf_ok(in, nbytes, p, leaf_lut)) {
          const uint32_t idx = atomicAdd(&L->n2, 1u);
          if (idx < kFindFull) L->c2[idx] = (uint32_t)(p - g0);
        }
      }
      __syncwarp();
    }
    const uint32_t n2 = L->n2;
    if (n2 > kFindFull) {
      // (rare: more survivors than the list holds) the lane-by-lane search
      // from this group on gives the same answer
      __syncwarp();
      return warp_find_first(in, nbytes, g0, to, hi_to, lane, out_lo, out_hi, leaf_lut, nullptr);
    }
    uint64_t best = kNoStop;
    for (uint32_t j = lane; j < n2; j += 32) {
      const uint64_t p = g0 + L->c2[j];
      if (p < best && dyn_candidate_full(in, nbytes, p)) best = p;
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) best = min(best, __shfl_xor_sync(0xFFFFFFFFu, best, d));
    __syncwarp();
    if (best != kNoStop) {
      out_lo = out_hi = best;
      return true;
    }
    if (have && best_lo < g1) break;
  }
  out_lo = best_lo;
  out_hi = best_hi;
  return have;
}

static __device__ bool warp_find_first(const uint8_t* __restrict__ in, uint64_t nbytes,
                                       uint64_t from, uint64_t to, uint64_t hi_to, int lane,
                                       uint64_t& out_lo, uint64_t& out_hi,
                                       const uint16_t* leaf_lut, FinderLists* L, bool dyn_only) {
  if (L)
    return warp_find_first_grouped(in, nbytes, from, to, hi_to, lane, out_lo, out_hi, leaf_lut, L,
                                   dyn_only);
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  if (to > nbytes * 8) to = nbytes * 8;
  if (hi_to > nbytes * 8) hi_to = nbytes * 8;
  bool have = false;
  uint64_t best_lo = 0, best_hi = 0;
  const uint64_t until = nbytes >= 5 ? min((hi_to + 7) / 8, nbytes - 4) : 0;
  uint64_t next_off = max((from + 3 + 7) / 8, (uint64_t)2);
  for (uint64_t w0 = from; w0 < to; w0 += 1024) {
    const uint64_t w1 = min(w0 + 1024, to);
    // stored offsets whose candidate may start below w1 (start >= off*8 - 10)
    const uint64_t off_end = min(until, (w1 + 10) / 8 + 1);
    while (!have && next_off < off_end) {
      const uint64_t ob = next_off + 4 * (uint64_t)lane;
      uint32_t m = 0;
      if (ob < off_end) {
        m = stored_filter4(bits64_at(in32, ob * 8));
        if (ob + 4 > off_end) m &= (1u << (off_end - ob)) - 1;
      }
      uint64_t lo = 0, hi = 0;
      bool hit = false;
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        if (stored_candidate(in, nbytes, ob + k, from, to, hi_to, lo, hi)) {
          hit = true;
          break;
        }
      }
      const uint32_t b = __ballot_sync(0xFFFFFFFFu, hit);
      if (b) {
        const int src = __ffs(b) - 1;
        best_lo = __shfl_sync(0xFFFFFFFFu, lo, src);
        best_hi = __shfl_sync(0xFFFFFFFFu, hi, src);
        have = true;
      }
      next_off = min(next_off + 128, off_end);
    }
    // dynamic candidates below the stored one (a tie at its bit_offset sorts first)
    const uint64_t lim = have ? min(w1, best_lo + 1) : w1;
    const uint64_t pl = w0 + 32 * (uint64_t)lane;
    uint32_t m = 0;
    if (pl < lim) {
      m = dyn_filter32(bits64_at(in32, pl));
      if (pl + 32 > lim) m &= (1u << (lim - pl)) - 1;
    }
    int hit = -1;
    while (m) {
      const int i = __ffs(m) - 1;
      m &= m - 1;
      if (dyn_candidate_fast(in, nbytes, pl + i, leaf_lut)) {
        hit = i;
        break;
      }
    }
    const uint32_t b = __ballot_sync(0xFFFFFFFFu, hit >= 0);
    if (b) {
      const int src = __ffs(b) - 1;
      const int i = __shfl_sync(0xFFFFFFFFu, hit, src);
      out_lo = out_hi = w0 + 32 * (uint64_t)src + (uint64_t)i;
      return true;
    }
    if (have && best_lo < w1) break;
  }
  out_lo = best_lo;
  out_hi = best_hi;
  return have;
}

// ---------------------------------------------------------------------------
// Sync starts in fixed-Huffman data (no counterpart in the reference, whose
// finder has no fixed-Huffman candidates: a fixed block has no header to
// test).  A walk decodes only positions with the fixed code of RFC 1951
// 3.2.6: a literal/length code, a length's extra bits, the 5-bit distance
// code and its extra bits; EOB must be followed by another fixed-block
// header.  Walks from a true symbol boundary never fail and all reach the
// same first boundary at or past the target; walks from a wrong bit fail
// (codes 286-287, distance codes 30-31, a non-fixed header) or fall into
// step with the true boundaries.  The search walks kSyncOffsets start bits
// and takes the end position most walks agree on (at least two; ties go to
// the lower position).  Whether that position really is a boundary is
// decided by the predecessor chunk, which hands over only on reaching it as
// a symbol start inside a non-final fixed block.
// ---------------------------------------------------------------------------
static __constant__ uint8_t f_len_extra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                               2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
static __constant__ uint8_t f_dist_extra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                                6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

// k <= 25 bits at absolute bit p from staged words sw (sw[0] = input word wbase)
static __device__ __forceinline__ uint32_t staged_bits(const uint32_t* sw, uint64_t wbase,
                                                       uint64_t p, int k) {
  const uint32_t i = (uint32_t)((p >> 5) - wbase), sh = (uint32_t)(p & 31);
  const uint64_t v = (((uint64_t)sw[i + 1] << 32) | sw[i]) >> sh;
  return (uint32_t)v & ((1u << k) - 1);
}

// first symbol boundary >= target of the fixed-code walk from p, or kSyncFail
static __device__ uint64_t fixed_walk(const uint32_t* sw, uint64_t wbase, uint64_t p,
                                      uint64_t target) {
  while (p < target) {
    const uint32_t x = staged_bits(sw, wbase, p, 9);
    const uint32_t c7 = __brev(x & 127u) >> 25, c8 = __brev(x & 255u) >> 24;
    uint32_t sym;
    if (c7 <= 0x17) {
      sym = 256 + c7;
      p += 7;
    } else if (c8 <= 0xBF) {
      sym = c8 - 0x30;
      p += 8;
    } else if (c8 <= 0xC7) {
      sym = 280 + (c8 - 0xC0);
      p += 8;
    } else {
      sym = 144 + ((__brev(x) >> 23) - 0x190);
      p += 9;
    }
    if (sym < 256) continue;
    if (sym == 256) {
      if ((staged_bits(sw, wbase, p, 3) >> 1) != 1) return kSyncFail;
      p += 3;
      continue;
    }
    if (sym > 285) return kSyncFail;
    p += f_len_extra[sym - 257];
    const uint32_t dc = __brev(staged_bits(sw, wbase, p, 5)) >> 27;
    if (dc >= 30) return kSyncFail;
    p += 5 + f_dist_extra[dc];
  }
  return p;
}

// words a sync search from `from` stages: [from >> 5, (target + 96) >> 5] + 1
constexpr uint32_t kSyncWords = (uint32_t)((kSyncOffsets + kSyncSpan + 96 + 64) / 32) + 2;

// ---------------------------------------------------------------------------
// Expected output bytes per compressed byte of the dynamic block whose header
// starts at `bit` (a candidate the finder accepted), from its code lengths
// alone: a code of length L stands for a symbol of probability 2^-L.
// Literals give one byte, a length symbol its mean length; a symbol costs its
// code, its extra bits and, for a length, the mean distance code and extra
// bits.  Used to cut high-ratio partitions finer (no reference counterpart).
// ---------------------------------------------------------------------------
static __constant__ uint16_t f_len_base[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,
                                               15, 17, 19, 23, 27, 31, 35, 43, 51,  59,
                                               67, 83, 99, 115, 131, 163, 195, 227, 258};

static __device__ __noinline__ float dyn_header_ratio(const uint8_t* in, uint64_t nbytes,
                                                      uint64_t bit) {
  const uint32_t h = (uint32_t)peek_bits(in, nbytes, bit, 17);
  const int hl = 257 + ((h >> 3) & 31), hd = 1 + ((h >> 8) & 31), pc = ((h >> 13) & 15) + 4;
  const uint64_t pbits = peek_bits(in, nbytes, bit + 17, 3 * pc);
  uint8_t cl[19];
  for (int i = 0; i < 19; i++) cl[i] = 0;
  for (int i = 0; i < pc; i++) cl[f_cl_order[i]] = (uint8_t)((pbits >> (3 * i)) & 7);
  uint16_t cnt[8], first[8], offs[8];
  uint8_t sorted[19];
  for (int L = 0; L < 8; L++) cnt[L] = 0;
  for (int s = 0; s < 19; s++) cnt[cl[s]]++;
  cnt[0] = 0;
  {
    uint32_t code = 0, off = 0;
    for (int L = 1; L < 8; L++) {
      if (L > 1) code = (code + cnt[L - 1]) << 1;
      first[L] = (uint16_t)code;
      offs[L] = (uint16_t)off;
      off += cnt[L];
    }
    uint16_t nx[8];
    for (int L = 0; L < 8; L++) nx[L] = offs[L];
    for (int s = 0; s < 19; s++)
      if (cl[s]) sorted[nx[cl[s]]++] = (uint8_t)s;
  }
  float out = 0.f, bits = 0.f, len_p = 0.f, dist_bits = 0.f, dist_p = 0.f;
  uint64_t pos = bit + 17 + 3 * pc;
  const int total = hl + hd;
  uint32_t prev = 0;
  for (int i = 0; i < total;) {
    const uint32_t rev = __brev((uint32_t)peek_bits(in, nbytes, pos, 14)) >> 25;
    int sym = -1;
    for (int L = 1; L < 8; L++) {
      const uint32_t idx = (rev >> (7 - L)) - first[L];
      if (idx < cnt[L]) {
        sym = sorted[offs[L] + idx];
        pos += L;
        break;
      }
    }
    if (sym < 0) return 0.f;
    uint32_t v = (uint32_t)sym;
    int rep = 1;
    if (sym == 16) {
      v = prev;
      rep = 3 + (int)peek_bits(in, nbytes, pos, 2);
      pos += 2;
    } else if (sym == 17) {
      v = 0;
      rep = 3 + (int)peek_bits(in, nbytes, pos, 3);
      pos += 3;
    } else if (sym == 18) {
      v = 0;
      rep = 11 + (int)peek_bits(in, nbytes, pos, 7);
      pos += 7;
    }
    if (v) {
      const float p = __int_as_float((127 - (int)v) << 23);  // 2^-v
      for (int k = i; k < i + rep && k < total; k++) {
        if (k < 256) {
          out += p;
          bits += p * (float)v;
        } else if (k >= 257 && k < hl && k < 286) {
          const int li = k - 257;
          len_p += p;
          out += p * ((float)f_len_base[li] + 0.5f * (float)((1u << f_len_extra[li]) - 1));
          bits += p * (float)(v + f_len_extra[li]);
        } else if (k >= hl) {
          const int di = k - hl;
          if (di < 30) {
            dist_p += p;
            dist_bits += p * (float)(v + f_dist_extra[di]);
          }
        }
      }
    }
    prev = v;
    i += rep;
  }
  if (dist_p > 0.f) bits += len_p * dist_bits / dist_p;
  return bits > 0.f ? 8.f * out / bits : 0.f;
}

}  // namespace gzgpu

