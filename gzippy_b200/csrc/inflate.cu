// inflate.cu -- speculative chunk inflate (RFC 1951) for sm_100a.
//
// One warp decodes one chunk.  All 32 lanes run the serial Huffman decode in
// lock-step on identical state (table reads are shared-memory broadcasts and
// control flow never diverges); the lanes split the work that is parallel:
// LZ77 copies (32 entries per step), stored-block copies and table builds.
//
// Entries are u16: a byte (< 256), or a window marker (>= 32768) for a
// back-reference that reaches before the chunk into the unknown 32 KiB
// window: window index w = 32768 + pos - dist gives the entry 32768 + w; a
// copy of a marker stays a marker.  This is the marker scheme of the
// reference (src/decompress/parallel/marker_inflate.rs init_marker_zone
// :265, replace_markers.rs:7-23).  A member's first chunk reads zeros there
// instead (the zero window of chunk_fetcher.rs:696).
//
// Two history layouts, same decode:
//   pages (default) : the chunk writes its entries straight into its output
//                     pages in HBM and reads back-references from them; a
//                     warp keeps only its Huffman tables (~7 KB) in shared
//                     memory, so an SM runs ~32 decoding warps and hides the
//                     latency of the serial symbol chain across them.
//   ring            : a 32 Ki-entry u16 ring per warp in shared memory
//                     (64 KB), flushed to the pages in 8 Ki-entry units;
//                     on-chip history, 3 decoding warps per SM.
//
// Stop rule (chunk_decode.rs decode_chunk :225): before each block header,
// stop if the bit position is >= stop_lo; the BFINAL block ends the chunk.
// A speculative chunk that fails moves on to its partition's next candidate
// (chunk_fetcher.rs speculative_decode_find_boundary :2616-2740).
//
// Input bits come from a two-window register stage: every lane holds one
// 32-bit word of the current and the next 128-byte input window; the bit
// buffer refills by warp shuffle, and the next window's load is issued a
// full window ahead of use.
#include <cstdint>

#include "common.cuh"
#include "finder_core.cuh"
#include "inflate.cuh"

namespace gzgpu {

__constant__ uint16_t c_len_base[29] = {3,  4,  5,  6,  7,  8,  9,  10,  11,  13,
                                        15, 17, 19, 23, 27, 31, 35, 43,  51,  59,
                                        67, 83, 99, 115, 131, 163, 195, 227, 258};
__constant__ uint8_t c_len_extra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                        2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__constant__ uint16_t c_dist_base[32] = {1,    2,    3,    4,    5,    7,     9,     13,
                                         17,   25,   33,   49,   65,   97,    129,   193,
                                         257,  385,  513,  769,  1025, 1537,  2049,  3073,
                                         4097, 6145, 8193, 12289, 16385, 24577, 0,     0};
__constant__ uint8_t c_dist_extra[32] = {0, 0, 0, 0, 1, 1, 2,  2,  3,  3,  4,  4,  5,  5, 6, 6,
                                         7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 0, 0};
__constant__ uint8_t c_cl_order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// litlen / dist table entry: [3:0] code length (0 = longer than the LUT or
// invalid), [7:4] extra bits, [9:8] kind, [31:16] literal / base value.
enum : uint32_t { kKindLit = 0, kKindLen = 1, kKindEob = 2, kKindBad = 3 };

__device__ __forceinline__ uint32_t litlen_entry(uint32_t sym, uint32_t L) {
  if (sym < 256) return (sym << 16) | (kKindLit << 8) | L;
  if (sym == 256) return (kKindEob << 8) | L;
  if (sym <= 285) {
    uint32_t k = sym - 257;
    return ((uint32_t)c_len_base[k] << 16) | ((uint32_t)c_len_extra[k] << 4) | (kKindLen << 8) | L;
  }
  return (kKindBad << 8) | L;
}
__device__ __forceinline__ uint32_t dist_entry(uint32_t sym, uint32_t L) {
  if (sym < 30) return ((uint32_t)c_dist_base[sym] << 16) | ((uint32_t)c_dist_extra[sym] << 4) | L;
  return (kKindBad << 8) | L;
}
__device__ __forceinline__ uint32_t pre_entry(uint32_t sym, uint32_t L) { return (sym << 16) | L; }

// 64-bit steps: entries of a step with matches staged in shared memory
// (larger steps write their pages directly)
constexpr uint32_t kWideStage = 256;

// Per-warp Huffman tables (shared memory).
template <int LB>
struct alignas(16) Tables {
  uint32_t lit_lut[1 << LB];
  uint32_t dist_lut[1 << kDistBits];
  uint16_t lit_sorted[288];
  uint16_t dist_sorted[32];
  uint16_t lit_count[16], lit_first[16], lit_offs[16];
  uint16_t dist_count[16], dist_first[16], dist_offs[16];
  uint16_t pre_count[16], pre_first[16], pre_offs[16];
  uint16_t next[16];
  union {
    struct {  // a block header's code lengths (read_tables only)
      uint32_t pre_lut[128];
      uint16_t pre_sorted[20];
      uint8_t lens[320];
    };
    struct {                       // 64-bit steps (huff_block_wide only)
      uint16_t stage[kWideStage];  // the entries of a step with matches
      uint8_t succ[64];            // a literal's successor bit per step bit (0xFF: other)
      uint16_t succ2[64];          // succ, and in the high byte the successor's succ (0xFF: none)
    };
  };
  uint8_t smap[32];  // output pass: lane of the symbol starting at each entry
  float p_len;       // the block's code space taken by length codes (sum of 2^-length)
};

template <int LB>
struct alignas(16) RingSmem {
  uint16_t ring[kWindow];
  Tables<LB> t;
};

// ---------------------------------------------------------------------------
// Bit reader over the register-staged input windows: a 128-bit bit window
// (bb = bits 0..63, hi = bits 64..127), refilled to > 96 valid bits.
// ---------------------------------------------------------------------------
struct BitReader {
  const uint32_t* in32;
  uint64_t win_base;  // word index of the current input window
  uint32_t win_cur;   // this lane's word of the current input window
  uint32_t win_next;  // this lane's word of the next input window
  uint64_t bb, hi;    // bit window (LSB = next bit)
  int bc;             // valid bits in the window
  uint64_t wpos;      // word index of the next word to append
  uint64_t limit_words;

  __device__ __forceinline__ void load_windows(uint64_t base, int lane) {
    win_base = base;
    win_cur = in32[base + lane];
    win_next = in32[base + 32 + lane];
  }
  __device__ __forceinline__ uint32_t word(uint64_t wi, int lane) {
    uint64_t rel = wi - win_base;
    if (rel >= 32) {
      if (rel < 64) {
        win_base += 32;
        win_cur = win_next;
        win_next = in32[win_base + 32 + lane];
      } else {
        load_windows(wi & ~31ull, lane);
      }
      rel = wi - win_base;
    }
    return __shfl_sync(0xFFFFFFFFu, win_cur, (int)rel);
  }
  __device__ __forceinline__ void seek(uint64_t bit, int lane) {
    uint64_t wi = bit >> 5;
    if (wi < win_base || wi >= win_base + 32) load_windows(wi & ~31ull, lane);
    bb = word(wi, lane) >> (bit & 31);
    hi = 0;
    bc = 32 - (int)(bit & 31);
    wpos = wi + 1;
  }
  __device__ __forceinline__ void append(uint32_t w) {
    if (bc < 64) {
      bb |= (uint64_t)w << bc;
      if (bc > 32) hi |= (uint64_t)w >> (64 - bc);
    } else {
      hi |= (uint64_t)w << (bc - 64);
    }
    bc += 32;
  }
  __device__ __forceinline__ void refill(int lane) {
    while (bc <= 96) append(word(wpos++, lane));
  }
  __device__ __forceinline__ void consume(int k) {  // 0 <= k < 64
    if (k) {
      bb = (bb >> k) | (hi << (64 - k));
      hi >>= k;
      bc -= k;
    }
  }
  __device__ __forceinline__ void consume_wide(int k) {  // 0 <= k < 128
    if (k >= 64) {
      bb = hi >> (k - 64);
      hi = 0;
      bc -= k;
    } else {
      consume(k);
    }
  }
  // bits [i, i + 64) of the window, 0 <= i < 64
  __device__ __forceinline__ uint64_t peek_at(int i) const {
    return i ? (bb >> i) | (hi << (64 - i)) : bb;
  }
  __device__ __forceinline__ uint64_t pos() const { return wpos * 32 - (uint64_t)bc; }
  __device__ __forceinline__ bool overrun() const { return wpos > limit_words; }
};

// ---------------------------------------------------------------------------
// Canonical Huffman table build, warp-cooperative.  lens[0..n) in shared.
// Acceptance follows zlib: over-subscribed sets fail; incomplete sets pass
// only when the longest code is one bit or the set is empty.
// ---------------------------------------------------------------------------
template <int TB, typename EntryFn>
__device__ bool build_table(const uint8_t* lens, int n, uint16_t* count, uint16_t* first,
                            uint16_t* offs, uint16_t* sorted, uint16_t* next, uint32_t* lut,
                            int lane, EntryFn entry) {
  // histogram by ballots: lane L (1..15) accumulates count[L]
  uint32_t cnt_l = 0;
  for (int g = 0; g < n; g += 32) {
    int s = g + lane;
    uint32_t l = s < n ? lens[s] : 0;
#pragma unroll
    for (int L = 1; L <= 15; L++) {
      uint32_t m = __ballot_sync(0xFFFFFFFFu, l == (uint32_t)L);
      if (lane == L) cnt_l += __popc(m);
    }
  }
  if (lane >= 1 && lane <= 15) count[lane] = (uint16_t)cnt_l;
  if (lane == 0) count[0] = 0;
  __syncwarp();
  // first code / offsets, validity (every lane computes the same values)
  int left = 1, maxl = 0;
  uint32_t code = 0, off = 0;
  for (int L = 1; L <= 15; L++) {
    uint32_t c = count[L];
    left = (left << 1) - (int)c;
    if (c) maxl = L;
    if (L > 1) code = (code + count[L - 1]) << 1;
    if (lane == L) {
      first[L] = (uint16_t)code;
      offs[L] = (uint16_t)off;
      next[L] = (uint16_t)off;
    }
    off += c;
    if (left < 0) break;
  }
  bool ok = left >= 0 && !(maxl > 0 && left > 0 && maxl != 1);
  __syncwarp();
  if (!ok) return false;
  // symbols sorted by (length, symbol)
  for (int g = 0; g < n; g += 32) {
    int s = g + lane;
    uint32_t l = s < n ? lens[s] : 0;
    uint32_t peers = __match_any_sync(0xFFFFFFFFu, l);
    uint32_t rank = __popc(peers & ((1u << lane) - 1));
    if (l) sorted[next[l] + rank] = (uint16_t)s;
    __syncwarp();
    if (l && (__ffs(peers) - 1) == lane) next[l] = (uint16_t)(next[l] + __popc(peers));
    __syncwarp();
  }
  // primary LUT: entry i decodes the code whose bits (LSB-first) are i
  for (int i = lane; i < (1 << TB); i += 32) {
    uint32_t rev = __brev((uint32_t)i) >> (32 - TB);  // MSB-first code bits
    uint32_t e = 0;
    for (int L = 1; L <= TB; L++) {
      uint32_t c = rev >> (TB - L);
      uint32_t idx = c - first[L];
      if (idx < count[L]) {
        e = entry(sorted[offs[L] + idx], (uint32_t)L);
        break;
      }
    }
    lut[i] = e;
  }
  __syncwarp();
  return true;
}

// Codes longer than the LUT: canonical first-code search on 15 bits.
// Returns the entry, or 0 for an invalid code.
template <int TB, typename EntryFn>
__device__ __forceinline__ uint32_t slow_decode(uint64_t bb, const uint16_t* count,
                                                const uint16_t* first, const uint16_t* offs,
                                                const uint16_t* sorted, EntryFn entry) {
  uint32_t rev = __brev((uint32_t)bb) >> 17;  // 15 code bits, first bit = MSB
  for (int L = TB + 1; L <= 15; L++) {
    uint32_t c = rev >> (15 - L);
    uint32_t idx = c - first[L];
    if (idx < count[L]) return entry(sorted[offs[L] + idx], (uint32_t)L);
  }
  return 0;
}

// Fixed (btype 1) or dynamic (btype 2) block tables; the 3 header bits are
// already consumed.  Returns kOk or an error status.
template <int LB>
__device__ int32_t read_tables(BitReader& br, uint32_t btype, Tables<LB>* T, uint64_t trunc_words,
                               int lane) {
  bool ok;
  if (btype == 1) {
    // fixed Huffman (RFC 1951 3.2.6): litlen 0..287, then 32 distance codes
    for (int s = lane; s < 320; s += 32) {
      uint8_t l;
      if (s < 144) l = 8;
      else if (s < 256) l = 9;
      else if (s < 280) l = 7;
      else if (s < 288) l = 8;
      else l = 5;
      T->lens[s] = l;
    }
    __syncwarp();
    ok = build_table<LB>(T->lens, 288, T->lit_count, T->lit_first, T->lit_offs, T->lit_sorted,
                         T->next, T->lit_lut, lane, litlen_entry);
    ok = ok && build_table<kDistBits>(T->lens + 288, 32, T->dist_count, T->dist_first,
                                      T->dist_offs, T->dist_sorted, T->next, T->dist_lut, lane,
                                      dist_entry);
    if (lane == 0) T->p_len = 24.f / 128.f + 6.f / 256.f;  // codes 256-279: 7 bits, 280-287: 8
    __syncwarp();
    return ok ? kOk : kBadDeflate;
  }
  // dynamic header (RFC 1951 3.2.7)
  br.refill(lane);
  uint32_t h = (uint32_t)br.bb & 0x3FFF;
  br.consume(14);
  int nlen = 257 + (h & 31), ndist = 1 + ((h >> 5) & 31), ncl = 4 + (h >> 10);
  if (nlen > 286 || ndist > 30) return kBadDeflate;
  // code-length code lengths: 3 bits each, read as up to 10 + 9
  uint32_t clv = 0;
  int n1 = ncl < 10 ? ncl : 10;
  br.refill(lane);
  if (lane < n1) clv = (uint32_t)(br.bb >> (3 * lane)) & 7;
  br.consume(3 * n1);
  br.refill(lane);
  if (lane >= 10 && lane < ncl) clv = (uint32_t)(br.bb >> (3 * (lane - 10))) & 7;
  br.consume(3 * (ncl - n1));
  if (lane < 19) T->lens[296 + c_cl_order[lane]] = (uint8_t)clv;
  __syncwarp();
  ok = build_table<7>(T->lens + 296, 19, T->pre_count, T->pre_first, T->pre_offs, T->pre_sorted,
                      T->next, T->pre_lut, lane, pre_entry);
  if (!ok) return kBadDeflate;
  int i = 0, total = nlen + ndist;
  uint32_t prev = 0;
  while (i < total) {
    br.refill(lane);
    if (br.overrun()) {
      ok = false;
      break;
    }
    uint32_t e = T->pre_lut[br.bb & 127];
    uint32_t L = e & 15;
    if (L == 0) {
      ok = false;
      break;
    }
    uint32_t sym = e >> 16;
    br.consume(L);
    if (sym < 16) {
      if (lane == 0) T->lens[i] = (uint8_t)sym;
      prev = sym;
      i++;
      continue;
    }
    int rep;
    uint32_t v = 0;
    if (sym == 16) {
      if (i == 0) {
        ok = false;
        break;
      }
      v = prev;
      rep = 3 + (int)(br.bb & 3);
      br.consume(2);
    } else if (sym == 17) {
      rep = 3 + (int)(br.bb & 7);
      br.consume(3);
    } else {
      rep = 11 + (int)(br.bb & 127);
      br.consume(7);
    }
    if (i + rep > total) {
      ok = false;
      break;
    }
    for (int j = lane; j < rep; j += 32) T->lens[i + j] = (uint8_t)v;
    prev = v;
    i += rep;
  }
  __syncwarp();
  if (br.overrun()) return br.wpos > trunc_words ? kTruncated : kOvershoot;
  if (!ok || T->lens[256] == 0) return kBadDeflate;
  // the code space of the length codes (257 .. nlen-1): a literal-heavy
  // block has little (the block decoder is chosen by it)
  {
    const int sym = 257 + lane;
    const uint32_t L = sym < nlen ? T->lens[sym] : 0u;
    float w = L ? __uint_as_float((127u - L) << 23) : 0.f;  // 2^-L
#pragma unroll
    for (int d = 16; d; d >>= 1) w += __shfl_xor_sync(0xFFFFFFFFu, w, d);
    if (lane == 0) T->p_len = w;
  }
  // the dist lengths must not alias the precode area: move them to 288+
  uint8_t dl = lane < ndist ? T->lens[nlen + lane] : 0;
  __syncwarp();
  T->lens[288 + lane] = lane < ndist ? dl : 0;
  __syncwarp();
  ok = build_table<LB>(T->lens, nlen, T->lit_count, T->lit_first, T->lit_offs, T->lit_sorted,
                       T->next, T->lit_lut, lane, litlen_entry);
  ok = ok && build_table<kDistBits>(T->lens + 288, ndist, T->dist_count, T->dist_first,
                                    T->dist_offs, T->dist_sorted, T->next, T->dist_lut, lane,
                                    dist_entry);
  return ok ? kOk : kBadDeflate;
}

// ---------------------------------------------------------------------------
// Page allocation (both layouts).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t alloc_page(const PagePool& pool, uint32_t cid, uint32_t gen,
                                               uint32_t seq, int lane) {
  uint32_t p = 0;
  if (lane == 0) {
    p = atomicAdd(pool.next, 1u);
    if (p < pool.cap) {
      pool.owner[p] = cid;
      pool.seq[p] = (gen << kGenShift) | seq;
    }
  }
  p = __shfl_sync(0xFFFFFFFFu, p, 0);
  return p < pool.cap ? p : kNoPage;
}

// ---------------------------------------------------------------------------
// History in the chunk's own pages.
//   seq s = index of the page holding the current output position o; the
//   pages of seq s-1, s, s+1 are kept in registers.  A back-reference reads
//   [o - 32768, o): seq s-1 or s.  A symbol writes [o, o + 258): seq s or s+1.
// ---------------------------------------------------------------------------
struct PageHist {
  uint16_t* data;
  uint32_t prev, cur, next;  // page ids of seq s-1, s, s+1 (kNoPage = none)
  uint64_t s;
  uint32_t n_pages;
  bool failed;

  __device__ __forceinline__ uint16_t* at(uint64_t q) const {
    uint64_t qs = q >> 16;
    uint32_t pg = qs == s ? cur : (qs < s ? prev : next);
    return data + (size_t)pg * kPageEntries + (q & (kPageEntries - 1));
  }
  __device__ __forceinline__ uint32_t page_of_seq(uint64_t x) const {
    return x == s ? cur : (x + 1 == s ? prev : (x == s + 1 ? next : kNoPage));
  }
  // make positions [o, o_end) writable (o_end - o <= kPageEntries)
  __device__ __forceinline__ bool ensure(const PagePool& pool, uint32_t cid, uint32_t gen,
                                         uint64_t o_end, int lane) {
    if (cur == kNoPage) {
      cur = alloc_page(pool, cid, gen, (uint32_t)s, lane);
      n_pages++;
      if (cur == kNoPage) return failed = true, false;
    }
    if (((o_end - 1) >> 16) > s && next == kNoPage) {
      next = alloc_page(pool, cid, gen, (uint32_t)(s + 1), lane);
      n_pages++;
      if (next == kNoPage) return failed = true, false;
    }
    return true;
  }
  __device__ __forceinline__ void advance(uint64_t o) {
    if ((o >> 16) > s) {
      prev = cur;
      cur = next;
      next = kNoPage;
      s++;
    }
  }
};

// ---------------------------------------------------------------------------
// Ring history in shared memory, flushed to pages.
// ---------------------------------------------------------------------------
struct PageWriter {
  uint32_t page;  // current page (kNoPage before the first)
  uint32_t prev;  // previous page
  uint32_t fill;  // entries in the current page
  uint32_t n_pages;
  bool failed;

  __device__ __forceinline__ bool ensure(const PagePool& pool, uint32_t cid, uint32_t gen,
                                         int lane) {
    if (page != kNoPage && fill < kPageEntries) return true;
    uint32_t p = alloc_page(pool, cid, gen, n_pages, lane);
    if (p == kNoPage) return failed = true, false;
    prev = page;
    page = p;
    fill = 0;
    n_pages++;
    return true;
  }
};

__device__ __forceinline__ bool ring_flush_full(uint16_t* ring, PageWriter& pw,
                                                const PagePool& pool, uint64_t& flushed,
                                                uint32_t cid, uint32_t gen, int lane) {
  if (!pw.ensure(pool, cid, gen, lane)) return false;
  __syncwarp();
  const uint4* src = reinterpret_cast<const uint4*>(ring + ((uint32_t)flushed & kRingMask));
  uint4* dst = reinterpret_cast<uint4*>(pool.data + (size_t)pw.page * kPageEntries + pw.fill);
#pragma unroll 4
  for (int k = lane; k < (int)(kFlush / 8); k += 32) dst[k] = src[k];
  pw.fill += kFlush;
  flushed += kFlush;
  return true;
}

__device__ bool ring_flush_tail(const uint16_t* ring, PageWriter& pw, const PagePool& pool,
                                uint64_t& flushed, uint64_t o, uint32_t cid, uint32_t gen,
                                int lane) {
  __syncwarp();
  while (flushed < o) {
    if (!pw.ensure(pool, cid, gen, lane)) return false;
    uint32_t r = (uint32_t)(o - flushed);
    uint32_t room = kPageEntries - pw.fill;
    uint32_t k = r < room ? r : room;
    uint16_t* dst = pool.data + (size_t)pw.page * kPageEntries + pw.fill;
    for (uint32_t j = lane; j < k; j += 32) dst[j] = ring[((uint32_t)flushed + j) & kRingMask];
    pw.fill += k;
    flushed += k;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Huffman block body, lane-parallel (page history).
//
// Every step, lane i decodes a whole symbol as if one started at bit i of the
// window: the litlen code, its extra bits and, for a length, the distance
// code and its extra bits (<= 48 bits).  The symbols that really start in the
// first 32 bits form a chain 0 -> total(0) -> ... that a few warp shuffles
// walk; literals of the chain are stored in parallel at their prefix-sum
// output offsets, then the matches are copied in order, 32 entries per pass.
// One step replaces ~4-6 dependent table lookups by one parallel lookup and
// a shuffle per symbol.
// ---------------------------------------------------------------------------
constexpr uint32_t kStepMaxOut = 16 * 258 + 32;  // output bound of one step

// Decode the symbol at bits [0, 48) of x with the full tables (long codes
// included).  Returns packed info ([5:0] total bits, [7:6] kind, [31:16]
// literal or length); *dist gets the distance; kind kKindBad if invalid.
template <int LB>
__device__ __forceinline__ uint32_t decode_symbol_full(uint64_t x, const Tables<LB>* T,
                                                       uint32_t* dist) {
  constexpr uint32_t LMASK = (1u << LB) - 1, DMASK = (1u << kDistBits) - 1;
  uint32_t e = T->lit_lut[x & LMASK];
  if ((e & 15) == 0)
    e = slow_decode<LB>(x, T->lit_count, T->lit_first, T->lit_offs, T->lit_sorted, litlen_entry);
  if (e == 0) return kKindBad << 6;
  uint32_t L = e & 15, kind = (e >> 8) & 3, val = e >> 16, total = L;
  if (kind == kKindLen) {
    uint32_t xb = (e >> 4) & 15;
    val += (uint32_t)(x >> L) & ((1u << xb) - 1);
    uint32_t sh = L + xb;
    uint64_t y = x >> sh;
    uint32_t de = T->dist_lut[y & DMASK];
    if ((de & 15) == 0)
      de = slow_decode<kDistBits>(y, T->dist_count, T->dist_first, T->dist_offs, T->dist_sorted,
                                  dist_entry);
    if (de == 0 || ((de >> 8) & 3) == kKindBad) return kKindBad << 6;
    uint32_t DL = de & 15, dxb = (de >> 4) & 15;
    *dist = (de >> 16) + ((uint32_t)(y >> DL) & ((1u << dxb) - 1));
    total = sh + DL + dxb;
  }
  return total | (kind << 6) | (val << 16);
}

// Page of a position relative to the start of page seq s: prev / cur / next.
__device__ __forceinline__ uint16_t* page_addr(const PageHist& ph, int32_t rel) {
  const uint32_t pg = rel < 0 ? ph.prev : (rel < (int32_t)kPageEntries ? ph.cur : ph.next);
  return ph.data + (size_t)pg * kPageEntries + ((uint32_t)rel & (kPageEntries - 1));
}

// kSync: the successor checks for sync starts and for starts gone by
// mid-block (compiled out when the job has no sync starts)
template <int LB, bool kSync>
__device__ __forceinline__ int32_t huff_block_parallel(
    BitReader& br, const Tables<LB>* T, PageHist& ph_io, const PagePool& pool, uint32_t cid,
    uint32_t gen, uint64_t& o_io, uint64_t& guard_io, uint64_t& marker_end_io, bool zero_window,
    uint64_t trunc_words, uint64_t sync_target, uint64_t passed_bit, bool& synced, bool& passed,
    int lane) {
  constexpr uint32_t LMASK = (1u << LB) - 1, DMASK = (1u << kDistBits) - 1;
  // the loop state in registers, written back on return
  PageHist ph = ph_io;
  uint64_t o = o_io, guard = guard_io, marker_end = marker_end_io;
  uint64_t pos = br.pos();
  int32_t status = kOk;
  for (;;) {
    // the successor's sync start: stop exactly there if it is a symbol
    // start of this block; rt = its offset in this step (>= 32: not here)
    uint32_t rt = 1000;
    if (kSync && sync_target != kNoStop && sync_target >= pos) {
      if (sync_target == pos) {
        synced = true;
        break;
      }
      if (sync_target - pos < 32) rt = (uint32_t)(sync_target - pos);
    }
    if (o >= guard) {
      ph.advance(o);
      if (!ph.ensure(pool, cid, gen, o + kStepMaxOut, lane)) {
        status = kPoolExhausted;
        break;
      }
      uint64_t pe = (ph.s + 1) << 16;  // end of the current page
      guard = ph.next != kNoPage ? pe : pe - kStepMaxOut;
    }
    // the step's 128 bits, from the register-staged input words
    // (the header reader's read-ahead may have moved the staging past w0)
    const uint64_t w0 = pos >> 5;
    if (w0 < br.win_base || w0 + 3 >= br.win_base + 64) {
      if (w0 >= br.win_base && w0 < br.win_base + 64) {
        br.win_base += 32;
        br.win_cur = br.win_next;
        br.win_next = br.in32[br.win_base + 32 + lane];
      } else {
        br.load_windows(w0 & ~31ull, lane);
      }
    }
    if (w0 + 4 > br.limit_words) {
      status = w0 + 4 > trunc_words ? kTruncated : kOvershoot;
      break;
    }
    uint32_t W[4];
    {
      const uint32_t rel = (uint32_t)(w0 - br.win_base);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint32_t r = rel + k;
        const uint32_t a = __shfl_sync(0xFFFFFFFFu, br.win_cur, r & 31);
        const uint32_t b2 = __shfl_sync(0xFFFFFFFFu, br.win_next, r & 31);
        W[k] = r < 32 ? a : b2;
      }
    }
    // lane-local decode of a symbol starting at bit `lane` of the step
    const uint32_t t = (uint32_t)(pos & 31) + lane;  // 0..62
    const uint32_t wa = t >> 5, bsh = t & 31;
    const uint64_t lo64 = wa ? ((uint64_t)W[2] << 32 | W[1]) : ((uint64_t)W[1] << 32 | W[0]);
    const uint32_t hi32 = wa ? W[3] : W[2];
    const uint64_t x = bsh ? (lo64 >> bsh) | ((uint64_t)hi32 << (64 - bsh)) : lo64;
    uint32_t info, dinfo = 0;
    {
      uint32_t e = T->lit_lut[x & LMASK];
      uint32_t L = e & 15, kind = (e >> 8) & 3, val = e >> 16, total = L;
      uint32_t slow = L == 0;
      if (!slow && kind == kKindLen) {
        uint32_t xb = (e >> 4) & 15;
        val += (uint32_t)(x >> L) & ((1u << xb) - 1);
        uint32_t sh = L + xb;
        uint64_t y = x >> sh;
        uint32_t de = T->dist_lut[y & DMASK];
        uint32_t DL = de & 15;
        if (DL == 0 || ((de >> 8) & 3) == kKindBad) {
          slow = 1;  // long or invalid distance code: resolved on the chain
        } else {
          uint32_t dxb = (de >> 4) & 15;
          dinfo = (de >> 16) + ((uint32_t)(y >> DL) & ((1u << dxb) - 1));
          total = sh + DL + dxb;
        }
      }
      info = total | (kind << 6) | (slow << 8) | (val << 16);
    }
    // The chain: each lane packs the successor of a symbol starting at its
    // bit ([7:0]; 128 + lane when the symbol needs the full tables, ends the
    // block or is invalid) with the entries it writes ([16:8]).  Walking the
    // chain from bit 0 gives every symbol on it its output offset `excl`.
    const uint32_t kind0 = (info >> 6) & 3;
    const uint32_t pk = ((info & 0x100) || kind0 >= kKindEob)
                            ? 128u + lane
                            : (lane + (info & 63)) | ((kind0 == kKindLit ? 1u : (info >> 16)) << 8);
    uint32_t p = 0, acc = 0, excl = 0;
    bool on = false, eob = false, at_sync = false;
    for (;;) {
      const uint32_t v = __shfl_sync(0xFFFFFFFFu, pk, (int)p);
      if (lane == (int)p) {
        on = true;
        excl = acc;
      }
      if ((v & 0xFF) >= 128) {
        // the symbol at p with the full tables (the same in every lane)
        uint32_t dd = 0;
        const uint32_t ts = (uint32_t)(pos & 31) + p;
        const uint32_t was = ts >> 5, bs = ts & 31;
        const uint64_t l64 = was ? ((uint64_t)W[2] << 32 | W[1]) : ((uint64_t)W[1] << 32 | W[0]);
        const uint32_t h32 = was ? W[3] : W[2];
        const uint32_t ip =
            decode_symbol_full<LB>(bs ? (l64 >> bs) | ((uint64_t)h32 << (64 - bs)) : l64, T, &dd);
        if (lane == (int)p) {
          info = ip;
          dinfo = dd;
        }
        const uint32_t kd = (ip >> 6) & 3;
        if (kd == kKindBad) {
          status = kBadDeflate;
          break;
        }
        p += ip & 63;
        if (kd == kKindEob) {
          eob = true;
          break;
        }
        acc += kd == kKindLit ? 1u : (ip >> 16);
      } else {
        acc += v >> 8;
        p = v & 0xFF;
      }
      if (kSync && p == rt) {  // the walk ends at the successor's sync start
        at_sync = true;
        break;
      }
      if (p >= 32) break;
    }
    if (status != kOk) break;
    const uint32_t kind = (info >> 6) & 3;
    const bool is_match = on && kind == kKindLen;
    // a back-reference before the start of the 32 KiB window is invalid
    if (__any_sync(0xFFFFFFFFu, is_match && (uint64_t)dinfo > o + excl + kWindow)) {
      status = kBadDeflate;
      break;
    }
    const int32_t orel = (int32_t)(o - (ph.s << 16));  // o within page seq s
    if (!__any_sync(0xFFFFFFFFu, is_match)) {
      // literals only: one store each, at their offsets
      if (on && kind == kKindLit) *page_addr(ph, orel + (int32_t)excl) = (uint16_t)(info >> 16);
    } else {
      // The step's entries in passes of 32, lane i writing entry e0 + i: a
      // literal's value, or a match entry copied from `dist` entries back.
      // A source before this pass is read from the pages (or is a window
      // marker / zero before the chunk); a source inside the pass is taken
      // from its lane by pointer jumping (sources lie strictly below).
      const uint32_t olen = on ? (kind == kKindLit ? 1u : (kind == kKindLen ? (info >> 16) : 0u)) : 0u;
      uint8_t* smap = const_cast<uint8_t*>(T->smap);  // the warp's scratch beside its tables
      uint32_t carry = 0;  // lane of the symbol that covers the pass's first entry
      for (uint32_t e0 = 0; e0 < acc; e0 += 32) {
        const bool starts = olen && excl >= e0 && excl < e0 + 32;
        const uint32_t smask = __reduce_or_sync(0xFFFFFFFFu, starts ? 1u << (excl - e0) : 0u);
        if (starts) smap[excl - e0] = (uint8_t)lane;
        __syncwarp();
        const uint32_t below = smask & (0xFFFFFFFFu >> (31 - lane));
        const uint32_t L = below ? smap[31 - __clz(below)] : carry;
        carry = __shfl_sync(0xFFFFFFFFu, L, 31);
        const uint32_t iL = __shfl_sync(0xFFFFFFFFu, info, (int)L);
        const uint32_t dL = __shfl_sync(0xFFFFFFFFu, dinfo, (int)L);
        const uint32_t e = e0 + lane;
        const bool act = e < acc;
        uint32_t v = iL >> 16;  // a literal's value
        int32_t ref = -1;
        if (act && ((iL >> 6) & 3) == kKindLen) {
          const int32_t rel = (int32_t)e - (int32_t)dL;  // source, relative to the step start
          if (rel >= (int32_t)e0) {
            ref = rel - (int32_t)e0;
          } else if ((int64_t)o + rel >= 0) {
            v = *page_addr(ph, orel + rel);
          } else {
            v = zero_window ? 0u : (uint32_t)((int64_t)(kMarkerBase + kWindow) + (int64_t)o + rel);
          }
        }
        while (__any_sync(0xFFFFFFFFu, ref >= 0)) {
          const uint32_t rv = __shfl_sync(0xFFFFFFFFu, v, ref & 31);
          const int32_t rr = __shfl_sync(0xFFFFFFFFu, ref, ref & 31);
          if (ref >= 0) {
            v = rv;
            ref = rr;
          }
        }
        if (act) *page_addr(ph, orel + (int32_t)e) = (uint16_t)v;
        if (!zero_window) {
          const uint32_t m = __ballot_sync(0xFFFFFFFFu, act && v >= kMarkerBase);
          if (m) marker_end = o + e0 + 32 - __clz(m);
        }
        __syncwarp();
      }
    }
    __syncwarp();
    o += acc;
    pos += p;
    if (at_sync) {
      synced = true;
      break;
    }
    if (eob) break;
    // the successor's start went by mid-block: it can never be handed over
    if (kSync && passed_bit < pos) {
      passed = true;
      break;
    }
  }
  br.seek(pos, lane);
  br.refill(lane);
  ph_io = ph;
  o_io = o;
  guard_io = guard;
  marker_end_io = marker_end;
  return status;
}

// ---------------------------------------------------------------------------
// Huffman block body, lane-parallel over 64-bit steps (page history).
//
// A step covers the symbols that start in the next 64 bits.  Lane i looks
// up the literal/length code at bits i and i + 32 of the step in the LUT
// only: a literal's successor is its start plus its code length, kept in a
// 64-entry shared table beside a second one holding each entry's
// successor's successor.  A walk from bit 0 follows literals two at a time
// through that table (one broadcast read and one branch per two literals);
// a length code (then its extra bits, distance code and distance extra
// bits), the end-of-block code, a code longer than the LUT or an invalid
// code is decoded on the walk by the whole warp from the same bits
// (shared-memory broadcasts).  Compared with huff_block_parallel, a step
// carries twice the bits and no lane decodes a distance for a position that
// is not on the chain.  The chain is a 64-bit mask of symbol starts, so each
// lane's output offset is a population count.  Literals go to their output
// offsets in parallel; a step with matches builds its entries in a shared
// stage, where every match entry maps to an entry before the match, and
// writes them out in coalesced stores (larger steps copy in passes of 32
// entries, sources inside a pass by pointer jumping).
// ---------------------------------------------------------------------------
constexpr uint32_t kWideMaxOut = 32 * 258 + 64;  // output bound of one step (>= 2 bits per match)
// adaptive choice: blocks whose length codes take less of the code space
// than this decode in 64-bit steps, the others (many matches) in 32-bit steps
constexpr float kWideMaxLenSpace = 0.3f;

template <int LB, bool kSync>
__device__ __forceinline__ int32_t huff_block_wide(
    BitReader& br, const Tables<LB>* T, PageHist& ph_io, const PagePool& pool, uint32_t cid,
    uint32_t gen, uint64_t& o_io, uint64_t& guard_io, uint64_t& marker_end_io, bool zero_window,
    uint64_t trunc_words, uint64_t sync_target, uint64_t passed_bit, bool& synced, bool& passed,
    int lane) {
  constexpr uint32_t LMASK = (1u << LB) - 1;
  PageHist ph = ph_io;
  uint64_t o = o_io, guard = guard_io, marker_end = marker_end_io;
  uint64_t pos = br.pos();
  int32_t status = kOk;
  for (;;) {
    uint32_t rt = 1000;  // the successor's sync start in this step (>= 64: not here)
    if (kSync && sync_target != kNoStop && sync_target >= pos) {
      if (sync_target == pos) {
        synced = true;
        break;
      }
      if (sync_target - pos < 64) rt = (uint32_t)(sync_target - pos);
    }
    // the step's 128 bits come from the register-staged input words; page,
    // window and limit checks share one branch in the common case
    const uint64_t w0 = pos >> 5;
    if (o >= guard || w0 - br.win_base > 60 || w0 + 4 > br.limit_words) {
      if (o >= guard) {
        ph.advance(o);
        if (!ph.ensure(pool, cid, gen, o + kWideMaxOut, lane)) {
          status = kPoolExhausted;
          break;
        }
        const uint64_t pe = (ph.s + 1) << 16;  // end of the current page
        guard = ph.next != kNoPage ? pe : pe - kWideMaxOut;
      }
      if (w0 < br.win_base || w0 + 3 >= br.win_base + 64) {
        if (w0 >= br.win_base && w0 < br.win_base + 64) {
          br.win_base += 32;
          br.win_cur = br.win_next;
          br.win_next = br.in32[br.win_base + 32 + lane];
        } else {
          br.load_windows(w0 & ~31ull, lane);
        }
      }
      if (w0 + 4 > br.limit_words) {
        status = w0 + 4 > trunc_words ? kTruncated : kOvershoot;
        break;
      }
    }
    uint32_t W[4];
    {
      const uint32_t rel = (uint32_t)(w0 - br.win_base);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint32_t r = rel + k;
        const uint32_t a = __shfl_sync(0xFFFFFFFFu, br.win_cur, r & 31);
        const uint32_t b2 = __shfl_sync(0xFFFFFFFFu, br.win_next, r & 31);
        W[k] = r < 32 ? a : b2;
      }
    }
    const uint32_t sh0 = (uint32_t)(pos & 31);
    // lane candidates at step bits lane and lane + 32: 32 bits each
    uint32_t val0, val1;
    uint8_t* succ = const_cast<uint8_t*>(T->succ);
    uint16_t* succ2 = const_cast<uint16_t*>(T->succ2);
    {
      const uint32_t t = sh0 + lane;  // 0..62
      const uint32_t wa = t >> 5, bs = t & 31;
      const uint32_t lo0 = wa ? W[1] : W[0], mid = wa ? W[2] : W[1], hi1 = wa ? W[3] : W[2];
      const uint32_t x0 = __funnelshift_r(lo0, mid, bs);
      const uint32_t x1 = __funnelshift_r(mid, hi1, bs);
      const uint32_t e0 = T->lit_lut[x0 & LMASK], e1 = T->lit_lut[x1 & LMASK];
      // a literal: its successor (step bit, < 128); anything else: 0xFF
      // (decoded on the walk by the whole warp)
      const uint32_t a0 = ((e0 & 15) && ((e0 >> 8) & 3) == kKindLit) ? lane + (e0 & 15) : 0xFFu;
      const uint32_t a1 = ((e1 & 15) && ((e1 >> 8) & 3) == kKindLit) ? lane + 32 + (e1 & 15) : 0xFFu;
      succ[lane] = (uint8_t)a0;
      succ[lane + 32] = (uint8_t)a1;
      val0 = e0 >> 16;
      val1 = e1 >> 16;
      __syncwarp();
      // two hops: the walk takes two literals per table read
      const uint32_t b0 = a0 < 64 ? succ[a0] : 0xFFu, b1 = a1 < 64 ? succ[a1] : 0xFFu;
      succ2[lane] = (uint16_t)(a0 | b0 << 8);
      succ2[lane + 32] = (uint16_t)(a1 | b1 << 8);
    }
    __syncwarp();
    // The walk: chain = the step bits where symbols on the chain from bit 0
    // start.  Literals are followed through the successor table (one
    // shared-memory broadcast each, no branch but the loop's); anything
    // else is decoded by the whole warp, and a match's extra entries
    // (length - 1) are counted for the lanes after it (corr).
    uint64_t chain = 0;
    uint32_t p = 0, corr0 = 0, corr1 = 0, corr = 0, d0 = 0, d1 = 0;
    bool m0 = false, m1 = false, any_m = false, eob = false, at_sync = false;
    for (;;) {
      uint32_t q;
      for (;;) {
        if (kSync && p == rt) {  // the walk ends at the successor's sync start
          at_sync = true;
          break;
        }
        // a = the literal at p's successor, b = a's (0xFF when a is not a
        // literal inside the step); one branch per two literals
        const uint32_t v = succ2[p], a = v & 0xFFu, b = v >> 8;
        if (b >= 64 || (kSync && a == rt)) {
          chain |= 1ull << p;
          if (a >= 64) {
            q = a;
          } else if (kSync && a == rt) {
            p = a;
            at_sync = true;
          } else {
            chain |= 1ull << a;
            p = a;
            q = b;
          }
          break;
        }
        chain |= (1ull << p) | (1ull << a);
        p = b;
      }
      if (at_sync) break;
      if (q < 0x80u) {  // a literal that ends past the step
        p = q;
        at_sync = kSync && p == rt;
        break;
      }
      // the whole symbol at step bit p, the same in every lane
      const uint32_t b = sh0 + p;  // bit in W, <= 94
      if (b + 48 > 128) {          // may not fit: the next step starts here
        chain &= ~(1ull << p);
        break;
      }
      const uint32_t wa = b >> 5, bs = b & 31;
      const uint64_t lo = wa == 0 ? ((uint64_t)W[1] << 32 | W[0])
                                  : (wa == 1 ? ((uint64_t)W[2] << 32 | W[1]) : ((uint64_t)W[3] << 32 | W[2]));
      const uint32_t h32 = wa == 0 ? W[2] : (wa == 1 ? W[3] : 0u);
      const uint64_t x = bs ? (lo >> bs) | ((uint64_t)h32 << (64 - bs)) : lo;
      uint32_t dist = 0;
      const uint32_t ip = decode_symbol_full<LB>(x, T, &dist);
      const uint32_t kd = (ip >> 6) & 3;
      if (kd == kKindBad) {
        status = kBadDeflate;
        break;
      }
      if (kd == kKindEob) {
        chain &= ~(1ull << p);
        p += ip & 63;
        eob = true;
        break;
      }
      const uint32_t acc_here = (uint32_t)__popcll(chain) - 1 + corr;  // entries before it
      // a back-reference before the start of the 32 KiB window is invalid
      if (kd == kKindLen && (uint64_t)dist > o + acc_here + kWindow) {
        status = kBadDeflate;
        break;
      }
      if (lane == (int)(p & 31)) {
        if (p >> 5) {
          m1 = kd == kKindLen; val1 = ip >> 16; d1 = dist;
        } else {
          m0 = kd == kKindLen; val0 = ip >> 16; d0 = dist;
        }
      }
      if (kd == kKindLen) {
        any_m = true;
        const uint32_t more = (ip >> 16) - 1;
        corr += more;
        corr0 += p < (uint32_t)lane ? more : 0u;
        corr1 += p < (uint32_t)lane + 32 ? more : 0u;
      }
      p += ip & 63;
      if (kSync && p == rt) {
        at_sync = true;
        break;
      }
      if (p >= 64) break;
    }
    if (status != kOk) break;
    // output offsets: symbols on the chain before the lane's bit, plus the
    // extra entries of the matches before it (the chain's two halves are
    // the two slots)
    const uint32_t c_lo = (uint32_t)chain, c_hi = (uint32_t)(chain >> 32);
    const uint32_t lt = (1u << lane) - 1;
    const uint32_t n_lo = __popc(c_lo);
    const uint32_t acc = n_lo + __popc(c_hi) + corr;
    const bool on0 = (c_lo >> lane) & 1, on1 = (c_hi >> lane) & 1;
    const uint32_t ex0 = __popc(c_lo & lt) + corr0;
    const uint32_t ex1 = n_lo + __popc(c_hi & lt) + corr1;
    const int32_t orel = (int32_t)(o - (ph.s << 16));  // o within page seq s
    if (!any_m) {
      // literals only: one store each, at their offsets
      if (orel + acc <= kPageEntries) {  // the step's entries lie in the current page
        uint16_t* base = ph.data + (size_t)ph.cur * kPageEntries + orel;
        if (on0) base[ex0] = (uint16_t)val0;
        if (on1) base[ex1] = (uint16_t)val1;
      } else {
        if (on0) *page_addr(ph, orel + (int32_t)ex0) = (uint16_t)val0;
        if (on1) *page_addr(ph, orel + (int32_t)ex1) = (uint16_t)val1;
      }
    } else if (acc <= kWideStage) {
      // The step's entries are built in the warp's shared stage, then go
      // to the pages in coalesced stores.  Literals first; then the matches
      // in chain order (slot-0 lanes, then slot-1 lanes).  Every entry of a
      // match maps to an entry before the match (final in the stage, or
      // history), so all its loads are in flight together.
      uint16_t* stage = const_cast<uint16_t*>(T->stage);
      if (on0 && !m0) stage[ex0] = (uint16_t)val0;
      if (on1 && !m1) stage[ex1] = (uint16_t)val1;
      __syncwarp();
      // an entry before the match: the stage, history, or before the chunk
      auto older = [&](int32_t src) -> uint32_t {
        if (src >= 0) return stage[src];
        if ((int64_t)o + src >= 0) return *page_addr(ph, orel + src);
        return zero_window ? 0u : (uint32_t)((int64_t)(kMarkerBase + kWindow) + (int64_t)o + src);
      };
      uint32_t mm0 = __ballot_sync(0xFFFFFFFFu, on0 && m0), mm1 = __ballot_sync(0xFFFFFFFFu, on1 && m1);
      while (mm0 | mm1) {
        const bool hi = mm0 == 0;
        const int l = __ffs(hi ? mm1 : mm0) - 1;
        if (hi) mm1 &= mm1 - 1;
        else mm0 &= mm0 - 1;
        const uint32_t mex = __shfl_sync(0xFFFFFFFFu, hi ? ex1 : ex0, l);
        const uint32_t mlen = __shfl_sync(0xFFFFFFFFu, hi ? val1 : val0, l);
        const uint32_t md = __shfl_sync(0xFFFFFFFFu, hi ? d1 : d0, l);
        // entry j of the match copies entry mex + j - md; for an overlapping
        // match (md < mlen) that source may lie inside the match, and
        // following it back by md at a time lands on mex - md + (j mod md)
        const bool overlap = md < mlen;
        for (uint32_t j0 = 0; j0 < mlen; j0 += 128) {
          uint32_t v[4];
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const uint32_t j = j0 + 32 * k + lane;
            const uint32_t jj = overlap ? j % md : j;
            v[k] = j < mlen ? older((int32_t)(mex + jj) - (int32_t)md) : 0u;
          }
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const uint32_t j = j0 + 32 * k + lane;
            if (j < mlen) stage[mex + j] = (uint16_t)v[k];
          }
        }
        __syncwarp();
      }
      for (uint32_t i0 = 0; i0 < acc; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool act = i < acc;
        const uint32_t v = act ? stage[i] : 0u;
        if (act) *page_addr(ph, orel + (int32_t)i) = (uint16_t)v;
        if (!zero_window) {
          const uint32_t m = __ballot_sync(0xFFFFFFFFu, act && v >= kMarkerBase);
          if (m) marker_end = o + i0 + 32 - __clz(m);
        }
      }
    } else {
      // The step's entries in passes of 32, lane i writing entry e0 + i: a
      // literal's value, or a match entry copied from `dist` entries back.
      // A symbol is named by (slot << 5) | lane; smap holds the one that
      // starts at each entry of the pass.
      uint8_t* smap = const_cast<uint8_t*>(T->smap);
      // packed per slot: value, bit 16 = match
      const uint32_t q0 = val0 | (m0 ? 0x10000u : 0u), q1 = val1 | (m1 ? 0x10000u : 0u);
      const uint32_t n0 = on0 ? (m0 ? val0 : 1u) : 0u, n1 = on1 ? (m1 ? val1 : 1u) : 0u;
      uint32_t carry = 0;  // symbol covering the pass's first entry
      for (uint32_t e0 = 0; e0 < acc; e0 += 32) {
        const bool s0 = n0 && ex0 >= e0 && ex0 < e0 + 32;
        const bool s1 = n1 && ex1 >= e0 && ex1 < e0 + 32;
        const uint32_t smask = __reduce_or_sync(
            0xFFFFFFFFu, (s0 ? 1u << (ex0 - e0) : 0u) | (s1 ? 1u << (ex1 - e0) : 0u));
        if (s0) smap[ex0 - e0] = (uint8_t)lane;
        if (s1) smap[ex1 - e0] = (uint8_t)(32 + lane);
        __syncwarp();
        const uint32_t below = smask & (0xFFFFFFFFu >> (31 - lane));
        const uint32_t S = below ? smap[31 - __clz(below)] : carry;
        carry = __shfl_sync(0xFFFFFFFFu, S, 31);
        const uint32_t qa = __shfl_sync(0xFFFFFFFFu, q0, (int)(S & 31));
        const uint32_t qb = __shfl_sync(0xFFFFFFFFu, q1, (int)(S & 31));
        const uint32_t da = __shfl_sync(0xFFFFFFFFu, d0, (int)(S & 31));
        const uint32_t db = __shfl_sync(0xFFFFFFFFu, d1, (int)(S & 31));
        const uint32_t qS = S >> 5 ? qb : qa, dS = S >> 5 ? db : da;
        const uint32_t e = e0 + lane;
        const bool act = e < acc;
        uint32_t v = qS & 0xFFFFu;  // a literal's value
        int32_t ref = -1;
        if (act && (qS >> 16)) {
          const int32_t rel = (int32_t)e - (int32_t)dS;  // source, relative to the step start
          if (rel >= (int32_t)e0) {
            ref = rel - (int32_t)e0;
          } else if ((int64_t)o + rel >= 0) {
            v = *page_addr(ph, orel + rel);
          } else {
            v = zero_window ? 0u : (uint32_t)((int64_t)(kMarkerBase + kWindow) + (int64_t)o + rel);
          }
        }
        while (__any_sync(0xFFFFFFFFu, ref >= 0)) {
          const uint32_t rv = __shfl_sync(0xFFFFFFFFu, v, ref & 31);
          const int32_t rr = __shfl_sync(0xFFFFFFFFu, ref, ref & 31);
          if (ref >= 0) {
            v = rv;
            ref = rr;
          }
        }
        if (act) *page_addr(ph, orel + (int32_t)e) = (uint16_t)v;
        if (!zero_window) {
          const uint32_t m = __ballot_sync(0xFFFFFFFFu, act && v >= kMarkerBase);
          if (m) marker_end = o + e0 + 32 - __clz(m);
        }
        __syncwarp();
      }
    }
    __syncwarp();
    o += acc;
    pos += p;
    if (at_sync) {
      synced = true;
      break;
    }
    if (eob) break;
    // the successor's start went by mid-block: it can never be handed over
    if (kSync && passed_bit < pos) {
      passed = true;
      break;
    }
  }
  br.seek(pos, lane);
  br.refill(lane);
  ph_io = ph;
  o_io = o;
  guard_io = guard;
  marker_end_io = marker_end;
  return status;
}

// ---------------------------------------------------------------------------
// Huffman block body, warp-uniform serial decode (page history).
//
// Every lane decodes the same symbol from the same bit window (table reads
// are shared-memory broadcasts), so a literal costs one table lookup and a
// few uniform ALU operations instead of 32 candidate decodes and a chain
// walk.  Output entries gather in lane registers: lane k holds entry wb + k
// of the current 32-entry aligned window (`cur`) and of the one before it
// (`prv`); a full window goes to the pages as one coalesced 64-byte store.
// A match fills the window lane-parallel: a source in `cur` or `prv` comes by
// shuffle, an older one from the pages, a source inside the entries being
// written by pointer jumping (sources lie strictly below their targets).
// ---------------------------------------------------------------------------
template <int LB, bool kSync>
__device__ __forceinline__ int32_t huff_block_serial(
    BitReader& br, const Tables<LB>* T, PageHist& ph_io, const PagePool& pool, uint32_t cid,
    uint32_t gen, uint64_t& o_io, uint64_t& guard_io, uint64_t& marker_end_io, bool zero_window,
    uint64_t trunc_words, uint64_t sync_target, uint64_t passed_bit, bool& synced, bool& passed,
    int lane) {
  constexpr uint32_t LMASK = (1u << LB) - 1, DMASK = (1u << kDistBits) - 1;
  int32_t status = kOk;
  // the loop state in registers, written back on return
  PageHist ph = ph_io;
  uint64_t o = o_io, guard = guard_io, marker_end = marker_end_io;
  auto done = [&](int32_t st) {
    ph_io = ph;
    o_io = o;
    guard_io = guard;
    marker_end_io = marker_end;
    return st;
  };
  if (o >= guard) {
    ph.advance(o);
    if (!ph.ensure(pool, cid, gen, o + kStepMaxOut, lane)) return done(kPoolExhausted);
    const uint64_t pe = (ph.s + 1) << 16;
    guard = ph.next != kNoPage ? pe : pe - kStepMaxOut;
  }
  // bit window: bits [pos, pos + bc) of the stream in bb, bc >= 32 before
  // each code; word wn is appended next
  const uint64_t pos0 = br.pos();
  uint64_t wn = pos0 >> 5;
  uint64_t bb = br.word(wn, lane) >> (pos0 & 31);
  int bc = 32 - (int)(pos0 & 31);
  wn++;
  // value of entry q < 0 (before the chunk): zero or its window marker
  auto before = [&](int64_t q) -> uint32_t {
    return zero_window ? 0u : (uint32_t)((int64_t)(kMarkerBase + kWindow) + q);
  };
  // the register windows, reloaded from the pages at block entry
  uint64_t wb = o & ~31ull;
  uint32_t cur = 0, prv = 0;
  {
    __syncwarp();
    if ((uint64_t)lane < o - wb) cur = *ph.at(wb + lane);
    const int64_t q = (int64_t)wb - 32 + lane;
    prv = q >= 0 ? (uint32_t)*ph.at((uint64_t)q) : before(q);
  }
  for (;;) {
    if (o >= guard) {
      ph.advance(o);
      if (!ph.ensure(pool, cid, gen, o + kStepMaxOut, lane)) {
        status = kPoolExhausted;
        break;
      }
      const uint64_t pe = (ph.s + 1) << 16;
      guard = ph.next != kNoPage ? pe : pe - kStepMaxOut;
    }
    if (kSync && wn * 32 - (uint64_t)bc == sync_target) {
      synced = true;
      break;
    }
    if (bc < 32) {
      if (wn + 3 > br.limit_words) {
        status = wn + 3 > trunc_words ? kTruncated : kOvershoot;
        break;
      }
      bb |= (uint64_t)br.word(wn, lane) << bc;
      bc += 32;
      wn++;
    }
    uint32_t e = T->lit_lut[bb & LMASK];
    if ((e & 15) == 0) {
      e = slow_decode<LB>(bb, T->lit_count, T->lit_first, T->lit_offs, T->lit_sorted, litlen_entry);
      if (e == 0) {
        status = kBadDeflate;
        break;
      }
    }
    const uint32_t L = e & 15, kind = (e >> 8) & 3;
    if (kind == kKindLit) {
      bb >>= L;
      bc -= (int)L;
      if ((uint64_t)lane == o - wb) cur = e >> 16;
      o++;
      if (o - wb == 32) {
        *ph.at(wb + lane) = (uint16_t)cur;
        prv = cur;
        wb += 32;
      }
      if (kSync && passed_bit < wn * 32 - (uint64_t)bc) {
        passed = true;
        break;
      }
      continue;
    }
    if (kind == kKindEob) {
      bb >>= L;
      bc -= (int)L;
      break;
    }
    if (kind == kKindBad) {
      status = kBadDeflate;
      break;
    }
    const uint32_t xb = (e >> 4) & 15;
    const uint32_t len = (e >> 16) + ((uint32_t)(bb >> L) & ((1u << xb) - 1));
    bb >>= L + xb;
    bc -= (int)(L + xb);
    if (bc < 32) {
      if (wn + 3 > br.limit_words) {
        status = wn + 3 > trunc_words ? kTruncated : kOvershoot;
        break;
      }
      bb |= (uint64_t)br.word(wn, lane) << bc;
      bc += 32;
      wn++;
    }
    uint32_t de = T->dist_lut[bb & DMASK];
    if ((de & 15) == 0) {
      de = slow_decode<kDistBits>(bb, T->dist_count, T->dist_first, T->dist_offs, T->dist_sorted,
                                  dist_entry);
      if (de == 0) {
        status = kBadDeflate;
        break;
      }
    }
    if (((de >> 8) & 3) == kKindBad) {
      status = kBadDeflate;
      break;
    }
    const uint32_t DL = de & 15, dxb = (de >> 4) & 15;
    const uint32_t dist = (de >> 16) + ((uint32_t)(bb >> DL) & ((1u << dxb) - 1));
    bb >>= DL + dxb;
    bc -= (int)(DL + dxb);
    if ((uint64_t)dist > o + kWindow) {
      status = kBadDeflate;
      break;
    }
    // LZ77 copy: entry o + j = entry o + j - dist, window by window
    for (uint32_t j0 = 0; j0 < len;) {
      const uint32_t k0 = (uint32_t)(o - wb);  // first free lane of the window
      const uint32_t n = min(32u - k0, len - j0);
      const bool act = (uint32_t)lane >= k0 && (uint32_t)lane < k0 + n;
      const int64_t src = (int64_t)wb + lane - (int64_t)dist;  // source of entry wb + lane
      uint32_t v = 0;
      int32_t ref = -1;  // a source among this pass's own entries: its lane
      const int64_t rel = src - (int64_t)wb;
      // an old source: from the pages (or before the chunk)
      const bool old = act && rel < -32;
      if (__any_sync(0xFFFFFFFFu, old)) {
        __syncwarp();
        if (old) v = src >= 0 ? (uint32_t)*ph.at((uint64_t)src) : before(src);
      }
      const uint32_t vc = __shfl_sync(0xFFFFFFFFu, cur, (int)(rel & 31));
      const uint32_t vp = __shfl_sync(0xFFFFFFFFu, prv, (int)(rel & 31));
      if (act && rel >= -32) {
        if (rel < 0) v = vp;
        else if (rel < (int64_t)k0) v = vc;
        else ref = (int32_t)rel;
      }
      while (__any_sync(0xFFFFFFFFu, ref >= 0)) {
        const uint32_t rv = __shfl_sync(0xFFFFFFFFu, v, ref & 31);
        const int32_t rr = __shfl_sync(0xFFFFFFFFu, ref, ref & 31);
        if (ref >= 0) {
          v = rv;
          ref = rr;
        }
      }
      if (act) cur = v;
      if (!zero_window) {
        const uint32_t m = __ballot_sync(0xFFFFFFFFu, act && v >= kMarkerBase);
        if (m) marker_end = wb + 32 - __clz(m);
      }
      o += n;
      j0 += n;
      if (o - wb == 32) {
        *ph.at(wb + lane) = (uint16_t)cur;
        prv = cur;
        wb += 32;
        __syncwarp();
      }
    }
    if (kSync && passed_bit < wn * 32 - (uint64_t)bc) {
      passed = true;
      break;
    }
  }
  // the open window's entries to the pages
  if ((uint64_t)lane < o - wb) *ph.at(wb + lane) = (uint16_t)cur;
  __syncwarp();
  br.seek(wn * 32 - (uint64_t)bc, lane);
  br.refill(lane);
  return done(status);
}

// ---------------------------------------------------------------------------
// Decode one chunk.  kRing selects the history layout.
// ---------------------------------------------------------------------------
// start bit a predecessor must reach to hand over to chunk k
__device__ __forceinline__ uint64_t handover_bit(const ChunkDesc& k) {
  return (k.flags & kChunkMemberFirst) ? k.limit_bit * 8 : k.lo_bit;
}

template <int LB, bool kRing, bool kSync>
__device__ int32_t decode_chunk(const uint8_t* __restrict__ in, ChunkDesc d,
                                const ChunkDesc* descs, ChunkResult* res, uint32_t cid,
                                uint32_t gen, uint16_t* ring, Tables<LB>* T,
                                const PagePool& pool, int lane) {
  const bool zero_window = (d.flags & kChunkMemberFirst) != 0;
  if (kRing) {
    // seed the ring: zeros for a member start, marker values otherwise
    for (uint32_t i = lane * 8; i < kWindow; i += 256) {
      uint4 v;
      if (zero_window) {
        v = make_uint4(0, 0, 0, 0);
      } else {
        uint32_t b = kMarkerBase + i;
        v.x = b | ((b + 1) << 16);
        v.y = (b + 2) | ((b + 3) << 16);
        v.z = (b + 4) | ((b + 5) << 16);
        v.w = (b + 6) | ((b + 7) << 16);
      }
      *reinterpret_cast<uint4*>(ring + i) = v;
    }
    __syncwarp();
  }

  BitReader br;
  br.in32 = reinterpret_cast<const uint32_t*>(in);
  // the window reads up to 128 bits (4 words) ahead of the decode position
  const uint64_t trunc_words = (d.in_end * 8 + 31) / 32 + 5;
  // the reader may run up to the abort bit (moved on by every extension)
  auto set_limit = [&]() {
    br.limit_words = (d.abort_bit != kNoStop && d.abort_bit / 32 + 5 < trunc_words)
                         ? d.abort_bit / 32 + 5
                         : trunc_words;
  };
  set_limit();
  br.load_windows((d.start_bit >> 5) & ~31ull, lane);
  br.seek(d.start_bit, lane);
  br.refill(lane);

  PageHist ph{pool.data, kNoPage, kNoPage, kNoPage, 0, 0, false};
  PageWriter pw{kNoPage, kNoPage, 0, 0, false};
  uint64_t o = 0, flushed = 0, marker_end = 0;
  uint32_t n_blocks = 0;
  int32_t status = kOk, final_block = 0;
  const uint64_t in_end_bits = d.in_end * 8;
  constexpr uint32_t LMASK = (1u << LB) - 1, DMASK = (1u << kDistBits) - 1;
  // page-history fast path: positions below `guard` need no page work
  uint64_t guard = 0;

  int extends = 0;
  const uint64_t slack = d.abort_bit != kNoStop ? d.abort_bit - d.stop_lo : 0;
  // a sync start begins inside a block: the Huffman block whose header is at
  // d.table_bit, or (table_bit 0) a non-final fixed-Huffman block
  bool in_sync_block = kSync && (d.flags & kChunkSync) != 0;
  bool synced = false;
  uint64_t blk_hdr = 0;  // header bit of the block being decoded (0 = unknown)
  uint32_t bfinal = 0, btype = 0;
  bool resume = false;  // continue the current block after going by a successor
  const bool confirmed = (d.flags & (kChunkMemberFirst | kChunkConfirmed)) != 0;
  // move on past successor d.next (a phantom) to nx_next, the chunk after it
  auto extend = [&](uint32_t nx_next) {
    if (nx_next == kNoChunk) {
      d.stop_lo = kNoStop;
      d.abort_bit = kNoStop;
    } else {
      d.stop_lo = handover_bit(descs[nx_next]);
      if (d.abort_bit != kNoStop) d.abort_bit = d.stop_lo + slack;
    }
    d.next = nx_next;
    extends++;
    set_limit();
  };
  for (;;) {
    uint64_t bitpos = br.pos();
    const bool resume_now = resume;
    resume = false;
    if (!resume_now && bitpos >= d.stop_lo) {
      // A block boundary past the successor's start range means that start
      // was a phantom: decode on to the start after it (the consumer's
      // re-decode from the confirmed boundary, chunk_fetcher.rs:855).
      if (d.next == kNoChunk) break;
      if (extends >= kMaxExtends && !(d.flags & (kChunkMemberFirst | kChunkConfirmed))) break;
      const ChunkDesc nx = descs[d.next];
      if (nx.flags & kChunkMemberFirst) break;
      // the successor's warp may have moved its start to a later candidate
      // (in-kernel retry) since this chunk's stop was set: read its range
      // afresh and keep decoding while still before it.  A stale or torn
      // read only costs a repair: the host walk checks every handover.
      const volatile ChunkDesc* vx = descs + d.next;
      const uint64_t nx_lo = vx->lo_bit, nx_start = vx->start_bit;
      if (bitpos < nx_lo) {
        d.stop_lo = nx_lo;
        if (d.abort_bit != kNoStop) d.abort_bit = d.stop_lo + slack;
        set_limit();
      } else {
        // a sync start is taken over only mid-block, at its exact symbol
        // start (huff_block_parallel); a block boundary at or past it
        // means this chunk went by it
        if (!(nx.flags & kChunkSync) && bitpos <= nx_start) break;
        if (nx.next == kNoChunk) {
          d.stop_lo = kNoStop;
          d.abort_bit = kNoStop;
        } else {
          d.stop_lo = handover_bit(descs[nx.next]);
          if (d.abort_bit != kNoStop) d.abort_bit = d.stop_lo + slack;
        }
        d.next = nx.next;
        extends++;
        set_limit();
        if (bitpos >= d.stop_lo) continue;
      }
    }
    if (resume_now) {
      // successors whose start this chunk is already past, mid-block
      while (d.next != kNoChunk && (confirmed || extends < kMaxExtends)) {
        if ((descs[d.next].flags & kChunkMemberFirst) ||
            ((const volatile ChunkDesc*)(descs + d.next))->start_bit >= bitpos)
          break;
        extend(descs[d.next].next);
      }
    }
    if (bitpos > d.abort_bit) {
      status = kOvershoot;
      break;
    }
    if (bitpos + 3 > in_end_bits) {
      status = kTruncated;
      break;
    }
    bool tables_ready = resume_now;
    if (resume_now) {
      // same block, tables in place
    } else if (in_sync_block) {
      in_sync_block = false;
      if (d.table_bit) {
        // the block's own header: type, BFINAL and code tables; then back
        // to the sync start
        br.seek(d.table_bit, lane);
        br.refill(lane);
        const uint32_t hdr = (uint32_t)br.bb & 7;
        br.consume(3);
        bfinal = hdr & 1;
        btype = hdr >> 1;
        if (btype != 1 && btype != 2) {
          status = kBadDeflate;
          break;
        }
        status = read_tables<LB>(br, btype, T, trunc_words, lane);
        if (status != kOk) break;
        tables_ready = true;
        blk_hdr = d.table_bit;
        br.seek(d.start_bit, lane);
        br.refill(lane);
      } else {
        bfinal = 0;
        btype = 1;
        blk_hdr = 0;
      }
    } else {
      blk_hdr = bitpos;
      if (pool.blocks && lane == 0) {
        const uint32_t k = atomicAdd(pool.n_blocks, 1u);
        if (k < pool.blocks_cap) pool.blocks[k] = BlockRec{bitpos, o, cid, gen};
      }
      br.refill(lane);
      const uint32_t hdr = (uint32_t)br.bb & 7;
      br.consume(3);
      bfinal = hdr & 1;
      btype = hdr >> 1;
    }
    if (btype == 0) {
      // stored block: byte-align, LEN/NLEN, raw copy
      br.consume(br.bc & 7);
      br.refill(lane);
      uint32_t ln = (uint32_t)br.bb & 0xFFFF, nln = (uint32_t)(br.bb >> 16) & 0xFFFF;
      br.consume(32);
      uint64_t byte = br.pos() >> 3;
      if (byte > d.in_end) {
        status = kTruncated;
        break;
      }
      if (ln != (~nln & 0xFFFFu)) {
        status = kBadDeflate;
        break;
      }
      if (byte + ln > d.in_end) {
        status = kTruncated;
        break;
      }
      uint32_t done = 0;
      while (done < ln) {
        uint32_t k = ln - done;
        if (k > 4096) k = 4096;
        const uint8_t* src = in + byte + done;
        if (kRing) {
          if (o - flushed >= kFlush && !ring_flush_full(ring, pw, pool, flushed, cid, gen, lane)) break;
          for (uint32_t j = lane; j < k; j += 32) ring[(uint32_t)(o + j) & kRingMask] = src[j];
        } else {
          ph.advance(o);
          if (!ph.ensure(pool, cid, gen, o + k, lane)) break;
          for (uint32_t j = lane; j < k; j += 32) *ph.at(o + j) = src[j];
        }
        o += k;
        done += k;
        __syncwarp();
      }
      if (pw.failed || ph.failed) {
        status = kPoolExhausted;
        break;
      }
      guard = 0;
      br.seek((byte + ln) * 8, lane);
    } else if (btype == 1 || btype == 2) {
      if (!tables_ready) status = read_tables<LB>(br, btype, T, trunc_words, lane);
      if (status != kOk) break;
      if (!kRing) {
        // the successor's sync start can be taken over only in the state
        // it assumes: inside its block (same header), or inside a non-final
        // fixed block for a fixed sync start.  Any successor whose start
        // goes by mid-block is a phantom (real starts are block boundaries
        // or sync starts reached exactly): the decode moves on past it.
        uint64_t sync_target = kNoStop, passed_bit = kNoStop;
        if (kSync && d.next != kNoChunk) {
          const ChunkDesc& nx = descs[d.next];
          if (nx.flags & kChunkSync) {
            const bool same = nx.table_bit ? (blk_hdr == nx.table_bit)
                                           : (btype == 1 && !bfinal);
            if (same) sync_target = nx.start_bit;
          }
          if (!(nx.flags & kChunkMemberFirst) && (confirmed || extends < kMaxExtends))
            passed_bit = ((const volatile ChunkDesc*)(descs + d.next))->start_bit;
        }
        bool passed = false;
        if (pool.serial == 1)
          status = huff_block_serial<LB, kSync>(br, T, ph, pool, cid, gen, o, guard, marker_end,
                                                zero_window, trunc_words, sync_target, passed_bit,
                                                synced, passed, lane);
        else if (pool.serial == 2 || (pool.serial == 3 && T->p_len < kWideMaxLenSpace))
          status = huff_block_wide<LB, kSync>(br, T, ph, pool, cid, gen, o, guard, marker_end,
                                              zero_window, trunc_words, sync_target, passed_bit,
                                              synced, passed, lane);
        else
          status = huff_block_parallel<LB, kSync>(br, T, ph, pool, cid, gen, o, guard, marker_end,
                                                  zero_window, trunc_words, sync_target, passed_bit,
                                                  synced, passed, lane);
        if (status != kOk || synced) break;
        if (passed) {
          extend(descs[d.next].next);
          resume = true;
          continue;
        }
        n_blocks++;
        if (bfinal) {
          final_block = 1;
          break;
        }
        continue;
      }
      // Huffman-coded block body (ring layout: serial decode)
      if constexpr (kRing) for (;;) {
        if (kRing) {
          if (o - flushed >= kFlush && !ring_flush_full(ring, pw, pool, flushed, cid, gen, lane)) {
            status = kPoolExhausted;
            break;
          }
        } else if (o >= guard) {
          ph.advance(o);
          if (!ph.ensure(pool, cid, gen, o + 258, lane)) {
            status = kPoolExhausted;
            break;
          }
          // o + 258 stays inside the mapped pages until o reaches guard
          uint64_t pe = (ph.s + 1) << 16;  // end of the current page
          guard = ph.next != kNoPage ? pe : pe - 258;
        }
        br.refill(lane);
        if (br.overrun()) {
          status = br.wpos > trunc_words ? kTruncated : kOvershoot;
          break;
        }
        uint32_t e = T->lit_lut[br.bb & LMASK];
        if ((e & 15) == 0) {
          e = slow_decode<LB>(br.bb, T->lit_count, T->lit_first, T->lit_offs, T->lit_sorted,
                              litlen_entry);
          if (e == 0) {
            status = kBadDeflate;
            break;
          }
        }
        uint32_t L = e & 15, kind = (e >> 8) & 3;
        if (kind == kKindLit) {
          br.consume(L);
          if (lane == 0) {
            if (kRing) ring[(uint32_t)o & kRingMask] = (uint16_t)(e >> 16);
            else *ph.at(o) = (uint16_t)(e >> 16);
          }
          o++;
          continue;
        }
        if (kind == kKindEob) {
          br.consume(L);
          break;
        }
        if (kind == kKindBad) {
          status = kBadDeflate;
          break;
        }
        uint32_t xb = (e >> 4) & 15;
        uint32_t len = (e >> 16) + (uint32_t)((br.bb >> L) & ((1u << xb) - 1));
        br.consume(L + xb);
        br.refill(lane);
        uint32_t de = T->dist_lut[br.bb & DMASK];
        if ((de & 15) == 0) {
          de = slow_decode<kDistBits>(br.bb, T->dist_count, T->dist_first, T->dist_offs,
                                      T->dist_sorted, dist_entry);
          if (de == 0) {
            status = kBadDeflate;
            break;
          }
        }
        if (((de >> 8) & 3) == kKindBad) {
          status = kBadDeflate;
          break;
        }
        uint32_t DL = de & 15, dxb = (de >> 4) & 15;
        uint32_t dist = (de >> 16) + (uint32_t)((br.bb >> DL) & ((1u << dxb) - 1));
        br.consume(DL + dxb);
        if ((uint64_t)dist > o + kWindow) {
          status = kBadDeflate;
          break;
        }
        // LZ77 copy: entry o+j = entry o-dist+(j mod dist); every source is
        // older than o, so the 32-wide steps are independent.
        __syncwarp();
        const bool wrap = dist < len;
        const uint32_t step_mod = wrap ? 32 % dist : 0;
        uint32_t r = wrap ? (uint32_t)lane % dist : (uint32_t)lane;  // j mod dist for j = lane
        for (uint32_t j0 = 0; j0 < len; j0 += 32) {
          const uint32_t j = j0 + lane;
          const bool act = j < len;
          uint16_t v = 0;
          if (act) {
            const uint32_t sj = wrap ? r : j;
            if (kRing) {
              v = ring[((uint32_t)o - dist + sj) & kRingMask];
              ring[((uint32_t)o + j) & kRingMask] = v;
            } else {
              const int64_t sp = (int64_t)o - (int64_t)dist + (int64_t)sj;
              if (sp >= 0) v = *ph.at((uint64_t)sp);
              else v = zero_window ? 0 : (uint16_t)(kMarkerBase + kWindow + sp);
              *ph.at(o + j) = v;
            }
          }
          if (!zero_window) {
            uint32_t m = __ballot_sync(0xFFFFFFFFu, act && v >= kMarkerBase);
            if (m) marker_end = o + j0 + 32 - __clz(m);
          }
          if (wrap) {
            r += step_mod;
            if (r >= dist) r -= dist;
          }
        }
        o += len;
      }
      if (status != kOk) break;
      __syncwarp();
    } else {
      status = kBadDeflate;
      break;
    }
    n_blocks++;
    if (bfinal) {
      final_block = 1;
      break;
    }
  }
  uint64_t end_bit = br.pos();
  if (status == kOk && end_bit > in_end_bits) status = kTruncated;
  uint32_t last_page = kNoPage, prev_page = kNoPage, n_pages = 0;
  if (kRing) {
    if (status == kOk && !ring_flush_tail(ring, pw, pool, flushed, o, cid, gen, lane)) status = kPoolExhausted;
    last_page = pw.page;
    prev_page = pw.prev;
    n_pages = pw.n_pages;
  } else {
    __syncwarp();
    if (o > 0) {
      ph.advance(o - 1);
      uint64_t ls = (o - 1) >> 16;
      last_page = ph.page_of_seq(ls);
      prev_page = ls > 0 ? ph.page_of_seq(ls - 1) : kNoPage;
    }
    n_pages = ph.n_pages;
  }
  if (lane == 0) {
    res->end_bit = end_bit;
    res->out_len = o;
    res->marker_end = marker_end;
    res->last_page = last_page;
    res->prev_page = prev_page;
    res->n_pages = n_pages;
    res->n_blocks = n_blocks;
    res->status = status;
    res->final_block = final_block;
    res->gen = gen;
    res->sync_end = synced ? 1u : 0u;
    res->end_hdr_bit = synced ? blk_hdr : 0;
  }
  __syncwarp();
  return status;
}

// Work loop shared by both kernels: take chunks from the queue; a failed
// speculative start moves on to the next candidate of its partition.
template <int LB, bool kRing, bool kSync>
__device__ __forceinline__ void work_loop(const uint8_t* __restrict__ in, ChunkDesc* descs,
                                          ChunkResult* results, const uint32_t* work,
                                          uint32_t n_work, uint32_t* work_counter,
                                          const PagePool& pool, uint16_t* ring, Tables<LB>* T,
                                          int lane) {
  for (;;) {
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(work_counter, 1u);
    w = __shfl_sync(0xFFFFFFFFu, w, 0);
    if (w >= n_work) break;
    uint32_t cid = work[w];
    ChunkDesc d = descs[cid];
    uint64_t t0 = 0;
    if (lane == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    const bool speculative =
        !(d.flags & (kChunkMemberFirst | kChunkSync)) && d.limit_bit > d.lo_bit;
    // attempts are numbered from the chunk's generation base (a chunk decoded
    // again after the page pool ran out tags its pages past the old ones)
    const uint32_t gen0 = d.flags >> kGenBaseShift;
    for (uint32_t gen = gen0;; gen++) {
      int32_t st = decode_chunk<LB, kRing, kSync>(in, d, descs, &results[cid], cid, gen, ring, T, pool,
                                           lane);
      if (st == kOk || st == kPoolExhausted || !speculative || gen + 1 >= gen0 + kMaxTries) break;
      uint64_t lo = 0, hi = 0;
      if (!warp_find_first(in, d.in_end, d.lo_bit + 1, d.limit_bit, d.limit_bit, lane, lo, hi)) break;
      d.lo_bit = lo;
      d.start_bit = hi;
      if (lane == 0) {
        descs[cid].lo_bit = lo;
        descs[cid].start_bit = hi;
      }
      __syncwarp();
    }
    if (lane == 0) {
      uint64_t t1;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
      results[cid].t_start = t0;
      results[cid].t_end = t1;
    }
  }
}

template <int LB>
__global__ void __launch_bounds__(32 * kRingWarps)
    inflate_ring_kernel(const uint8_t* __restrict__ in, ChunkDesc* __restrict__ descs,
                        ChunkResult* __restrict__ results, const uint32_t* __restrict__ work,
                        const uint32_t* __restrict__ n_work_ptr, uint32_t* work_counter,
                        PagePool pool) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  RingSmem<LB>* S = reinterpret_cast<RingSmem<LB>*>(smem) + warp;
  work_loop<LB, true, true>(in, descs, results, work, *n_work_ptr, work_counter, pool, S->ring,
                            &S->t, lane);
}

template <int LB, int MINB, bool kSync>
__global__ void __launch_bounds__(32 * kPageWarps, MINB)
    inflate_pages_kernel(const uint8_t* __restrict__ in, ChunkDesc* __restrict__ descs,
                         ChunkResult* __restrict__ results, const uint32_t* __restrict__ work,
                         const uint32_t* __restrict__ n_work_ptr, uint32_t* work_counter,
                         PagePool pool) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Tables<LB>* T = reinterpret_cast<Tables<LB>*>(smem) + warp;
  work_loop<LB, false, kSync>(in, descs, results, work, *n_work_ptr, work_counter, pool, nullptr,
                              T, lane);
}

template <int LB>
size_t inflate_smem_bytes(bool ring) {
  return ring ? sizeof(RingSmem<LB>) * kRingWarps : sizeof(Tables<LB>) * kPageWarps;
}

// page kernel instance for `ctas` CTAs per SM (registers sized for it), with
// or without sync-start support
template <int LB>
static const void* pages_kernel_fn(int ctas, bool sync) {
  if (sync)
    return ctas >= 4 ? (const void*)inflate_pages_kernel<LB, 4, true>
                     : (const void*)inflate_pages_kernel<LB, 3, true>;
  return ctas >= 4 ? (const void*)inflate_pages_kernel<LB, 4, false>
                   : (const void*)inflate_pages_kernel<LB, 3, false>;
}

template <int LB>
cudaError_t launch_inflate(bool ring, int ctas, bool sync, const uint8_t* in, ChunkDesc* descs,
                           ChunkResult* results, const uint32_t* work, const uint32_t* n_work,
                           uint32_t* work_counter, const PagePool& pool, int blocks,
                           cudaStream_t stream) {
  size_t smem = inflate_smem_bytes<LB>(ring);
  cudaError_t e;
  if (ring) {
    e = cudaFuncSetAttribute(inflate_ring_kernel<LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    inflate_ring_kernel<LB><<<blocks, 32 * kRingWarps, smem, stream>>>(in, descs, results, work,
                                                                       n_work, work_counter, pool);
  } else {
    const void* fn = pages_kernel_fn<LB>(ctas, sync);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&in,   (void*)&descs,        (void*)&results, (void*)&work,
                    (void*)&n_work, (void*)&work_counter, (void*)&pool};
    e = cudaLaunchKernel(fn, dim3(blocks), dim3(32 * kPageWarps), args, smem, stream);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

template <int LB>
int inflate_blocks_per_sm(bool ring, int ctas) {
  int n = 0;
  size_t smem = inflate_smem_bytes<LB>(ring);
  if (ring) {
    cudaFuncSetAttribute(inflate_ring_kernel<LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, inflate_ring_kernel<LB>, 32 * kRingWarps, smem);
  } else {
    // both variants are sized for the same registers; take the larger
    const void* fn = pages_kernel_fn<LB>(ctas, true);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, 32 * kPageWarps, smem);
    cudaFuncSetAttribute(pages_kernel_fn<LB>(ctas, false), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    if (n > ctas) n = ctas;
  }
  return n;
}

#define GZGPU_INST(LB)                                                                       \
  template size_t inflate_smem_bytes<LB>(bool);                                              \
  template int inflate_blocks_per_sm<LB>(bool, int);                                         \
  template cudaError_t launch_inflate<LB>(bool, int, bool, const uint8_t*, ChunkDesc*, ChunkResult*, \
                                          const uint32_t*, const uint32_t*, uint32_t*,       \
                                          const PagePool&, int, cudaStream_t);
GZGPU_INST(10)
GZGPU_INST(11)
GZGPU_INST(12)

// ---------------------------------------------------------------------------
// Sync starts inside dynamic blocks (no counterpart in the reference).  A
// partition (or piece) that the finder left without a start lies inside some
// block; the nearest regular start before it in its stream names that
// block's header (when a block start went unrecorded in between, the table is
// wrong, the walks fail or agree on a false start, and no predecessor ever
// hands over to it).  Warp 0 builds the block's code tables; each of
// the kSyncOffsets threads walks the code's symbol positions from one start
// bit to the first boundary at or past from + kSyncOffsets + kSyncSpanDyn
// (an EOB or an invalid code fails the walk); the end most walks agree on (at
// least two, ties to the lower bit) becomes the piece's start.  As with the
// fixed-code sync starts, the predecessor decides: it hands over only on
// reaching that bit as a symbol start inside the same block.
// ---------------------------------------------------------------------------
constexpr uint32_t kSyncScan = 256;  // chunks looked back for a block header

__global__ void __launch_bounds__(kSyncOffsets)
    dyn_sync_kernel(const uint8_t* __restrict__ in, ChunkDesc* descs,
                    const uint32_t* __restrict__ pieces, uint32_t n, uint32_t* n_sync) {
  constexpr int LB = 10;
  __shared__ Tables<LB> T;
  __shared__ uint64_t ends[kSyncOffsets];
  __shared__ uint64_t table;
  __shared__ int ok;
  if (blockIdx.x >= n) return;
  const uint32_t j = pieces[blockIdx.x];
  ChunkDesc& d = descs[j];
  if (d.flags & kChunkValid) return;
  const uint64_t from = d.guess_bit, to = d.limit_bit, nbytes = d.in_end;
  const uint64_t target = from + kSyncOffsets + kSyncSpanDyn;
  if (target + 64 > to || target + 128 > nbytes * 8) return;
  if (threadIdx.x == 0) {
    // nearest regular (non-sync) start before this range in its stream;
    // chunks other CTAs turn into sync starts meanwhile are skipped like the
    // invalid ones they were
    uint64_t t = 0;
    for (int64_t k = (int64_t)j - 1; k >= 0 && k + (int64_t)kSyncScan >= (int64_t)j; k--) {
      const ChunkDesc& p = descs[k];
      if (p.stream != d.stream) break;
      const uint32_t f = p.flags;
      if ((f & kChunkValid) && !(f & kChunkSync)) {
        if (p.start_bit < from && (peek_bits(in, p.in_end, p.start_bit, 3) >> 1) == 2)
          t = p.start_bit;
        break;
      }
    }
    table = t;
    ok = 0;
  }
  __syncthreads();
  if (!table) return;
  const int lane = threadIdx.x & 31;
  const uint64_t trunc_words = (nbytes * 8 + 31) / 32 + 5;
  if (threadIdx.x < 32) {
    BitReader br;
    br.in32 = reinterpret_cast<const uint32_t*>(in);
    br.limit_words = trunc_words;
    br.load_windows(((table + 3) >> 5) & ~31ull, lane);
    br.seek(table + 3, lane);
    br.refill(lane);
    const int32_t st = read_tables<LB>(br, 2, &T, trunc_words, lane);
    if (lane == 0) ok = st == kOk;
  }
  __syncthreads();
  if (!ok) return;
  uint64_t p = from + threadIdx.x, e = kSyncFail;
  while (p < target) {
    uint32_t dist = 0;
    const uint32_t info = decode_symbol_full<LB>(peek_bits(in, nbytes, p, 48), &T, &dist);
    const uint32_t kind = (info >> 6) & 3;
    if (kind == kKindBad || kind == kKindEob) break;
    p += info & 63;
    if (p >= target) e = p;
  }
  ends[threadIdx.x] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t best = kSyncFail;
    uint32_t best_n = 1;
    for (uint32_t i = 0; i < kSyncOffsets; i++) {
      const uint64_t v = ends[i];
      if (v == kSyncFail) continue;
      uint32_t c = 0;
      for (uint32_t k = 0; k < kSyncOffsets; k++) c += ends[k] == v;
      if (c > best_n || (c == best_n && best != kSyncFail && v < best)) {
        best = v;
        best_n = c;
      }
    }
    if (best != kSyncFail) {
      d.lo_bit = d.start_bit = best;
      d.table_bit = table;
      d.flags |= kChunkValid | kChunkSync;
      if (n_sync) atomicAdd(n_sync, 1u);
    }
  }
}

cudaError_t launch_dyn_sync(const uint8_t* in, ChunkDesc* descs, const uint32_t* pieces, uint32_t n,
                            uint32_t* n_sync, cudaStream_t stream) {
  if (!n) return cudaSuccess;
  dyn_sync_kernel<<<n, kSyncOffsets, 0, stream>>>(in, descs, pieces, n, n_sync);
  return cudaGetLastError();
}

// ===========================================================================
// Decode without allocating: gzgpu_decompress_device_noalloc.
//
// For callers that cannot call cudaMalloc -- code under a pool-only
// allocator that must not grow, real-time paths that cannot take the
// device-wide synchronisation cudaMalloc/cudaFree may cause, or processes
// whose device memory is reserved up front by another framework.  One warp decodes the stream's
// members one after another (no speculation) with the same page-history
// inflate as above; its pages, its chunk record and the status word live in
// one file-scope device array that every GPU loading this library holds
// until exit.  The caller owns input and output.
// ===========================================================================
constexpr uint64_t kNoAllocMaxOut = 4ull << 20;  // output limit of one call (bytes)
constexpr uint32_t kNoAllocPages = (uint32_t)(kNoAllocMaxOut / kPageEntries) + 2;

struct NoAllocScratch {
  int32_t status;
  uint32_t page_next;  // page allocation counter, cleared for every member
  uint64_t out_len;
  ChunkResult res;
  uint32_t owner[kNoAllocPages];
  uint32_t seq[kNoAllocPages];
  alignas(256) uint16_t pages[(size_t)kNoAllocPages * kPageEntries];
};

static __device__ __align__(256) uint8_t g_noalloc_scratch[sizeof(NoAllocScratch)];

static __device__ __forceinline__ uint32_t na_mulmod(uint32_t a, uint32_t b) {
  uint32_t r = 0;
  for (int i = 31; i >= 0; i--) {
    r ^= b & (0u - ((a >> i) & 1u));
    b = (b >> 1) ^ (0xEDB88320u & (0u - (b & 1u)));
  }
  return r;
}

// crc(A|B) from crc(A), crc(B) and |B|: x^(8|B|) * crc(A) + crc(B) mod P
static __device__ uint32_t na_crc_combine(uint32_t c1, uint32_t c2, uint64_t len2) {
  uint32_t xp = 1u << 30;  // x^1, squared up through x^(2^k)
  uint32_t p = 1u << 31;   // x^0
  for (uint64_t e = len2 * 8; e; e >>= 1) {
    if (e & 1) p = na_mulmod(xp, p);
    xp = na_mulmod(xp, xp);
  }
  return na_mulmod(p, c1) ^ c2;
}

// header length of the member at byte p of [0, n), 0 if malformed/truncated
static __device__ uint64_t na_header(const uint8_t* in, uint64_t p, uint64_t n) {
  if (n < p + 10 || in[p] != 0x1f || in[p + 1] != 0x8b || in[p + 2] != 8) return 0;
  uint8_t flg = in[p + 3];
  if (flg & 0xE0) return 0;
  uint64_t o = p + 10;
  if (flg & 4) {
    if (o + 2 > n) return 0;
    o += 2 + (in[o] | (in[o + 1] << 8));
    if (o > n) return 0;
  }
  for (int f = 8; f <= 16; f <<= 1)
    if (flg & f) {
      while (o < n && in[o]) o++;
      if (o >= n) return 0;
      o++;
    }
  if (flg & 2) o += 2;
  return o <= n ? o - p : 0;
}

__global__ void __launch_bounds__(32)
    noalloc_kernel(const uint8_t* __restrict__ in, uint64_t n, uint8_t* __restrict__ out,
                   uint64_t out_cap, NoAllocScratch* S) {
  __shared__ Tables<10> T;
  __shared__ uint32_t crc_tab[256];
  const int lane = threadIdx.x;
  for (uint32_t i = lane; i < 256; i += 32) {
    uint32_t c = i;
    for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
    crc_tab[i] = c;
  }
  __syncwarp();
  int32_t status = kOk;
  uint64_t total = 0, pos = 0;
  bool too_small = false;  // some member did not fit out_cap
  if (n < 2 || in[0] != 0x1f || in[1] != 0x8b) status = kNotGzip;
  for (uint32_t member = 0; status == kOk; member++) {
    if (member > 0 && (n - pos < 18 || in[pos] != 0x1f || in[pos + 1] != 0x8b)) break;
    const uint64_t hl = na_header(in, pos, n);
    if (hl == 0) {
      if (member == 0) status = (n < 10 || in[2] == 8) && !(n >= 10 && (in[3] & 0xE0)) ? kTruncated : kBadHeader;
      break;
    }
    ChunkDesc d{};
    d.start_bit = d.lo_bit = d.guess_bit = d.limit_bit = (pos + hl) * 8;
    d.stop_lo = kNoStop;
    d.abort_bit = kNoStop;
    d.in_end = n;
    d.flags = kChunkMemberFirst | kChunkValid;
    d.next = kNoChunk;
    if (lane == 0) S->page_next = 0;  // every member starts with an empty pool
    __syncwarp();
    const PagePool pool{S->pages, S->owner, S->seq, &S->page_next, kNoAllocPages};
    int32_t st = decode_chunk<10, false, false>(in, d, nullptr, &S->res, 0, 0, nullptr, &T, pool, lane);
    __syncwarp();
    const ChunkResult r = S->res;
    if (st == kPoolExhausted) {
      status = kNoAllocTooLarge;
      break;
    }
    if (st != kOk) {
      status = st;
      break;
    }
    if (!r.final_block) {
      status = kTruncated;
      break;
    }
    const uint64_t trailer = (r.end_bit + 7) / 8;
    if (trailer + 8 > n) {
      status = kTruncated;
      break;
    }
    if (total + r.out_len > kNoAllocMaxOut) {
      status = kNoAllocTooLarge;
      break;
    }
    // pages were taken in order, so entry q sits at pages[q] (no markers:
    // a member starts with the zero window).  Once a member does not fit
    // out_cap, later members are still decoded and checked, without being
    // written, so that *out_len reports the exact size needed.
    if (!too_small && total + r.out_len > out_cap) too_small = true;
    if (!too_small)
      for (uint64_t q = lane; q < r.out_len; q += 32) out[total + q] = (uint8_t)S->pages[q];
    __syncwarp();
    // CRC32 of the member's entries: each lane one slice, combined in order by lane 0
    const uint64_t per = (r.out_len + 31) / 32;
    const uint64_t b0 = min((uint64_t)lane * per, r.out_len), b1 = min(b0 + per, r.out_len);
    uint32_t c = 0xFFFFFFFFu;
    for (uint64_t q = b0; q < b1; q++) c = (c >> 8) ^ crc_tab[(c ^ (uint32_t)S->pages[q]) & 0xFF];
    c = ~c;
    uint32_t crc = 0;
    for (int l = 0; l < 32; l++) {
      uint32_t cl = __shfl_sync(0xFFFFFFFFu, c, l);
      uint64_t ll = min(per, r.out_len - min((uint64_t)l * per, r.out_len));
      if (lane == 0) crc = na_crc_combine(crc, cl, ll);
    }
    crc = __shfl_sync(0xFFFFFFFFu, crc, 0);
    const uint8_t* t = in + trailer;
    const uint32_t ecrc = t[0] | (t[1] << 8) | ((uint32_t)t[2] << 16) | ((uint32_t)t[3] << 24);
    const uint32_t eisz = t[4] | (t[5] << 8) | ((uint32_t)t[6] << 16) | ((uint32_t)t[7] << 24);
    if ((uint32_t)r.out_len != eisz) status = kSizeMismatch;
    else if (crc != ecrc) status = kCrcMismatch;
    total += r.out_len;
    pos = trailer + 8;
    if (pos >= n) break;
  }
  if (status == kOk && too_small) status = kOutTooSmall;
  if (lane == 0) {
    S->status = status;
    S->out_len = total;
  }
}

}  // namespace gzgpu

#include <mutex>

#include "../../include/gzgpu.h"

namespace {
// device address of the scratch array, looked up once per device
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};
}  // namespace

extern "C" int gzgpu_decompress_device_noalloc(const void* d_in, size_t in_len, void* d_out,
                                               size_t out_cap, size_t* out_len,
                                               void* cuda_stream) {
  using namespace gzgpu;
  if (!out_len || (!d_in && in_len) || (!d_out && out_cap)) return GZGPU_INVALID_ARGUMENT;
  *out_len = 0;
  if (reinterpret_cast<uintptr_t>(d_in) & 3) return GZGPU_INVALID_ARGUMENT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return GZGPU_DEVICE_ERROR;
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      // the array's host-side name is a stand-in; the kernel needs its device address
      if (cudaGetSymbolAddress(&g_noalloc_ptr[dev], g_noalloc_scratch) != cudaSuccess) {
        g_noalloc_ptr[dev] = nullptr;
        return GZGPU_DEVICE_ERROR;
      }
    }
    scratch = g_noalloc_ptr[dev];
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(cuda_stream);
  NoAllocScratch* S = reinterpret_cast<NoAllocScratch*>(scratch);
  // cudaLaunchKernel reports this launch's own failure; the thread's
  // last-error state, which may hold an earlier error of the caller's, is
  // neither read nor cleared
  const uint8_t* k_in = reinterpret_cast<const uint8_t*>(d_in);
  uint64_t k_n = in_len, k_cap = out_cap;
  uint8_t* k_out = reinterpret_cast<uint8_t*>(d_out);
  void* args[] = {(void*)&k_in, (void*)&k_n, (void*)&k_out, (void*)&k_cap, (void*)&S};
  if (cudaLaunchKernel((const void*)noalloc_kernel, dim3(1), dim3(32), args, 0, st) != cudaSuccess)
    return GZGPU_DEVICE_ERROR;
  struct {
    int32_t status;
    uint32_t pad;
    uint64_t out_len;
  } res{};
  if (cudaMemcpyAsync(&res, scratch, sizeof(res), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return GZGPU_DEVICE_ERROR;
  *out_len = res.out_len;
  if (res.status == kNotGzip) *out_len = 0;
  return res.status;
}
