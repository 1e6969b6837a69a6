// inflate.cu -- speculative chunk inflate (RFC 1951) for sm_100a.
//
// One warp decodes one chunk.  All 32 lanes run the serial Huffman decode in
// lock-step on identical state (so table reads are shared-memory broadcasts
// and control flow never diverges); the lanes split the work that is
// parallel: LZ77 copies (32 entries per step), stored-block copies, table
// builds and ring -> page flushes (16-byte vector stores).
//
// History lives on chip: a 32 Ki-entry u16 ring in shared memory per warp.
// A chunk that starts without a window pre-seeds the ring with marker values
// (entry i = 32768 + i), so a back-reference that reaches before the chunk
// copies the marker for the window byte it needs; copies of markers stay
// markers.  This is the marker scheme of the reference
// (src/decompress/parallel/marker_inflate.rs init_marker_zone :265,
// replace_markers.rs:7-23).  A member's first chunk seeds zeros instead
// (the zero window of chunk_fetcher.rs:696).
//
// Stop rule (chunk_decode.rs decode_chunk :225): before each block header,
// stop if the bit position is >= stop_lo; the BFINAL block ends the chunk.
//
// Input bits come from a two-window register stage: every lane holds one
// 32-bit word of the current and the next 128-byte input window; the bit
// buffer refills by warp shuffle, and the next window's load is issued a
// full window ahead of use.
#include <cstdint>

#include "common.cuh"
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

template <int LB>
struct alignas(16) WarpSmem {
  uint16_t ring[kWindow];       // decoded history (u16 entries)
  uint32_t lit_lut[1 << LB];
  uint32_t dist_lut[1 << kDistBits];
  uint32_t pre_lut[128];
  uint16_t lit_sorted[288];
  uint16_t dist_sorted[32];
  uint16_t pre_sorted[19];
  uint16_t lit_count[16], lit_first[16], lit_offs[16];
  uint16_t dist_count[16], dist_first[16], dist_offs[16];
  uint16_t pre_count[16], pre_first[16], pre_offs[16];
  uint16_t next[16];
  uint8_t lens[320];
};

// ---------------------------------------------------------------------------
// Bit reader over the register-staged input windows.
// ---------------------------------------------------------------------------
struct BitReader {
  const uint32_t* in32;
  uint64_t win_base;  // word index of the current window
  uint32_t win_cur;   // this lane's word of the current window
  uint32_t win_next;  // this lane's word of the next window
  uint64_t bb;        // bit buffer (LSB = next bit)
  int bc;             // valid bits in bb
  uint64_t wpos;      // word index of the next word to append to bb
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
    load_windows(wi & ~31ull, lane);
    bb = word(wi, lane) >> (bit & 31);
    bc = 32 - (int)(bit & 31);
    wpos = wi + 1;
  }
  __device__ __forceinline__ void refill(int lane) {
    if (bc <= 32) {
      bb |= (uint64_t)word(wpos, lane) << bc;
      bc += 32;
      wpos++;
    }
  }
  __device__ __forceinline__ void consume(int k) {
    bb >>= k;
    bc -= k;
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
  // histogram by ballots (no shared atomics on 16-bit words)
  uint32_t cnt_l = 0;  // lane l (1..15) accumulates count[l]
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

// ---------------------------------------------------------------------------
// Output pages
// ---------------------------------------------------------------------------
struct PageWriter {
  uint32_t page;       // current page (kNoPage before the first)
  uint32_t prev;       // previous page
  uint32_t fill;       // entries in the current page
  uint32_t n_pages;
  bool failed;

  __device__ __forceinline__ bool ensure(const PagePool& pool, uint32_t cid, int lane) {
    if (page != kNoPage && fill < kPageEntries) return true;
    uint32_t p = 0;
    if (lane == 0) {
      p = atomicAdd(pool.next, 1u);
      if (p < pool.cap) {
        pool.owner[p] = cid;
        pool.seq[p] = n_pages;
      }
    }
    p = __shfl_sync(0xFFFFFFFFu, p, 0);
    if (p >= pool.cap) {
      failed = true;
      return false;
    }
    prev = page;
    page = p;
    fill = 0;
    n_pages++;
    return true;
  }
};

template <int LB>
__device__ __forceinline__ bool flush_full(WarpSmem<LB>* S, PageWriter& pw, const PagePool& pool,
                                           uint64_t& flushed, uint32_t cid, int lane) {
  if (!pw.ensure(pool, cid, lane)) return false;
  __syncwarp();
  const uint4* src = reinterpret_cast<const uint4*>(S->ring + ((uint32_t)flushed & kRingMask));
  uint4* dst = reinterpret_cast<uint4*>(pool.data + (size_t)pw.page * kPageEntries + pw.fill);
#pragma unroll 4
  for (int k = lane; k < (int)(kFlush / 8); k += 32) dst[k] = src[k];
  pw.fill += kFlush;
  flushed += kFlush;
  return true;
}

template <int LB>
__device__ bool flush_tail(WarpSmem<LB>* S, PageWriter& pw, const PagePool& pool,
                           uint64_t& flushed, uint64_t o, uint32_t cid, int lane) {
  __syncwarp();
  while (flushed < o) {
    if (!pw.ensure(pool, cid, lane)) return false;
    uint32_t r = (uint32_t)(o - flushed);
    uint32_t room = kPageEntries - pw.fill;
    uint32_t k = r < room ? r : room;
    uint16_t* dst = pool.data + (size_t)pw.page * kPageEntries + pw.fill;
    for (uint32_t j = lane; j < k; j += 32) dst[j] = S->ring[((uint32_t)flushed + j) & kRingMask];
    pw.fill += k;
    flushed += k;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Decode one chunk.
// ---------------------------------------------------------------------------
template <int LB>
__device__ void decode_chunk(const uint8_t* __restrict__ in, const ChunkDesc& d, ChunkResult* res,
                             uint32_t cid, WarpSmem<LB>* S, const PagePool& pool, int lane) {
  const bool zero_window = (d.flags & kChunkMemberFirst) != 0;
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
    *reinterpret_cast<uint4*>(S->ring + i) = v;
  }
  __syncwarp();

  BitReader br;
  br.in32 = reinterpret_cast<const uint32_t*>(in);
  br.limit_words = (d.in_end * 8 + 31) / 32 + 2;
  br.seek(d.start_bit, lane);
  br.refill(lane);

  PageWriter pw{kNoPage, kNoPage, 0, 0, false};
  uint64_t o = 0, flushed = 0, marker_end = 0;
  uint32_t n_blocks = 0;
  int32_t status = kOk, final_block = 0;
  const uint64_t in_end_bits = d.in_end * 8;
  constexpr uint32_t LMASK = (1u << LB) - 1, DMASK = (1u << kDistBits) - 1;

  for (;;) {
    uint64_t bitpos = br.pos();
    if (bitpos >= d.stop_lo) break;
    if (bitpos + 3 > in_end_bits) {
      status = kTruncated;
      break;
    }
    br.refill(lane);
    uint32_t hdr = (uint32_t)br.bb & 7;
    br.consume(3);
    uint32_t bfinal = hdr & 1, btype = hdr >> 1;
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
        if (o - flushed >= kFlush) {
          if (!flush_full(S, pw, pool, flushed, cid, lane)) break;
        }
        uint32_t k = ln - done;
        if (k > 4096) k = 4096;
        const uint8_t* src = in + byte + done;
        for (uint32_t j = lane; j < k; j += 32) S->ring[(uint32_t)(o + j) & kRingMask] = src[j];
        o += k;
        done += k;
        __syncwarp();
      }
      if (pw.failed) {
        status = kPoolExhausted;
        break;
      }
      br.seek((byte + ln) * 8, lane);
    } else if (btype == 1 || btype == 2) {
      bool ok;
      if (btype == 1) {
        // fixed Huffman (RFC 1951 3.2.6)
        for (int s = lane; s < 320; s += 32) {
          uint8_t l;
          if (s < 144) l = 8;
          else if (s < 256) l = 9;
          else if (s < 280) l = 7;
          else if (s < 288) l = 8;
          else l = 5;  // 288..319: 32 distance codes of 5 bits
          S->lens[s] = l;
        }
        __syncwarp();
        ok = build_table<LB>(S->lens, 288, S->lit_count, S->lit_first, S->lit_offs, S->lit_sorted,
                             S->next, S->lit_lut, lane, litlen_entry);
        ok = ok && build_table<kDistBits>(S->lens + 288, 32, S->dist_count, S->dist_first,
                                          S->dist_offs, S->dist_sorted, S->next, S->dist_lut,
                                          lane, dist_entry);
      } else {
        // dynamic header (RFC 1951 3.2.7)
        br.refill(lane);
        uint32_t h = (uint32_t)br.bb & 0x3FFF;
        br.consume(14);
        int nlen = 257 + (h & 31), ndist = 1 + ((h >> 5) & 31), ncl = 4 + (h >> 10);
        if (nlen > 286 || ndist > 30) {
          status = kBadDeflate;
          break;
        }
        // code-length code lengths: 3 bits each, read as up to 10 + 9
        uint32_t clv = 0;
        int n1 = ncl < 10 ? ncl : 10;
        br.refill(lane);
        if (lane < n1) clv = (uint32_t)(br.bb >> (3 * lane)) & 7;
        br.consume(3 * n1);
        br.refill(lane);
        if (lane >= 10 && lane < ncl) clv = (uint32_t)(br.bb >> (3 * (lane - 10))) & 7;
        br.consume(3 * (ncl - n1));
        if (lane < 19) S->lens[296 + c_cl_order[lane]] = (uint8_t)clv;
        __syncwarp();
        ok = build_table<7>(S->lens + 296, 19, S->pre_count, S->pre_first, S->pre_offs,
                            S->pre_sorted, S->next, S->pre_lut, lane, pre_entry);
        if (!ok) {
          status = kBadDeflate;
          break;
        }
        int i = 0, total = nlen + ndist;
        uint32_t prev = 0;
        while (i < total) {
          br.refill(lane);
          if (br.overrun()) {
            ok = false;
            break;
          }
          uint32_t e = S->pre_lut[br.bb & 127];
          uint32_t L = e & 15;
          if (L == 0) {
            ok = false;
            break;
          }
          uint32_t sym = e >> 16;
          br.consume(L);
          if (sym < 16) {
            if (lane == 0) S->lens[i] = (uint8_t)sym;
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
          for (int j = lane; j < rep; j += 32) S->lens[i + j] = (uint8_t)v;
          prev = v;
          i += rep;
        }
        __syncwarp();
        if (!ok || S->lens[256] == 0 || br.overrun()) {
          status = br.overrun() ? kTruncated : kBadDeflate;
          break;
        }
        // the dist lengths must not alias the precode area: move them to 288+
        uint8_t dl = lane < ndist ? S->lens[nlen + lane] : 0;
        __syncwarp();
        if (lane < 32) S->lens[288 + lane] = lane < ndist ? dl : 0;
        __syncwarp();
        ok = build_table<LB>(S->lens, nlen, S->lit_count, S->lit_first, S->lit_offs, S->lit_sorted,
                             S->next, S->lit_lut, lane, litlen_entry);
        ok = ok && build_table<kDistBits>(S->lens + 288, ndist, S->dist_count, S->dist_first,
                                          S->dist_offs, S->dist_sorted, S->next, S->dist_lut,
                                          lane, dist_entry);
      }
      if (!ok) {
        status = kBadDeflate;
        break;
      }
      // Huffman-coded block body
      for (;;) {
        if (o - flushed >= kFlush) {
          if (!flush_full(S, pw, pool, flushed, cid, lane)) {
            status = kPoolExhausted;
            break;
          }
        }
        br.refill(lane);
        if (br.overrun()) {
          status = kTruncated;
          break;
        }
        uint32_t e = S->lit_lut[br.bb & LMASK];
        if ((e & 15) == 0) {
          e = slow_decode<LB>(br.bb, S->lit_count, S->lit_first, S->lit_offs, S->lit_sorted,
                              litlen_entry);
          if (e == 0) {
            status = kBadDeflate;
            break;
          }
        }
        uint32_t L = e & 15, kind = (e >> 8) & 3;
        if (kind == kKindLit) {
          br.consume(L);
          if (lane == 0) S->ring[(uint32_t)o & kRingMask] = (uint16_t)(e >> 16);
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
        uint32_t de = S->dist_lut[br.bb & DMASK];
        if ((de & 15) == 0) {
          de = slow_decode<kDistBits>(br.bb, S->dist_count, S->dist_first, S->dist_offs,
                                      S->dist_sorted, dist_entry);
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
        const uint32_t ob = (uint32_t)o;
        const bool wrap = dist < len;
        for (uint32_t j0 = 0; j0 < len; j0 += 32) {
          const uint32_t j = j0 + lane;
          const bool act = j < len;
          uint16_t v = 0;
          if (act) {
            uint32_t sj = wrap ? j % dist : j;
            v = S->ring[(ob - dist + sj) & kRingMask];
            S->ring[(ob + j) & kRingMask] = v;
          }
          if (!zero_window) {
            uint32_t m = __ballot_sync(0xFFFFFFFFu, act && v >= kMarkerBase);
            if (m) marker_end = o + j0 + 32 - __clz(m);
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
  if (status == kOk && !flush_tail(S, pw, pool, flushed, o, cid, lane)) status = kPoolExhausted;
  if (lane == 0) {
    res->end_bit = end_bit;
    res->out_len = o;
    res->marker_end = marker_end;
    res->last_page = pw.page;
    res->prev_page = pw.prev;
    res->n_pages = pw.n_pages;
    res->n_blocks = n_blocks;
    res->status = status;
    res->final_block = final_block;
  }
  __syncwarp();
}

template <int LB>
__global__ void __launch_bounds__(32 * kDecodeWarps)
    inflate_kernel(const uint8_t* __restrict__ in, const ChunkDesc* __restrict__ descs,
                   ChunkResult* __restrict__ results, const uint32_t* __restrict__ work,
                   const uint32_t* __restrict__ n_work_ptr, uint32_t* work_counter, PagePool pool) {
  const uint32_t n_work = *n_work_ptr;
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem<LB>* S = reinterpret_cast<WarpSmem<LB>*>(smem + warp * sizeof(WarpSmem<LB>));
  for (;;) {
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(work_counter, 1u);
    w = __shfl_sync(0xFFFFFFFFu, w, 0);
    if (w >= n_work) break;
    uint32_t cid = work[w];
    ChunkDesc d = descs[cid];
    decode_chunk<LB>(in, d, &results[cid], cid, S, pool, lane);
  }
}

template <int LB>
size_t inflate_smem_bytes() {
  return sizeof(WarpSmem<LB>) * kDecodeWarps;
}

template <int LB>
cudaError_t launch_inflate(const uint8_t* in, const ChunkDesc* descs, ChunkResult* results,
                           const uint32_t* work, const uint32_t* n_work, uint32_t* work_counter,
                           const PagePool& pool, int blocks, cudaStream_t stream) {
  size_t smem = inflate_smem_bytes<LB>();
  cudaError_t e = cudaFuncSetAttribute(inflate_kernel<LB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  inflate_kernel<LB><<<blocks, 32 * kDecodeWarps, smem, stream>>>(in, descs, results, work,
                                                                   n_work, work_counter, pool);
  return cudaGetLastError();
}

template <int LB>
int inflate_blocks_per_sm() {
  int n = 0;
  cudaFuncSetAttribute(inflate_kernel<LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)inflate_smem_bytes<LB>());
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, inflate_kernel<LB>, 32 * kDecodeWarps,
                                                inflate_smem_bytes<LB>());
  return n;
}

#define GZGPU_INST(LB)                                                                      \
  template size_t inflate_smem_bytes<LB>();                                                 \
  template int inflate_blocks_per_sm<LB>();                                                 \
  template cudaError_t launch_inflate<LB>(const uint8_t*, const ChunkDesc*, ChunkResult*,   \
                                          const uint32_t*, const uint32_t*, uint32_t*,      \
                                          const PagePool&, int, cudaStream_t);
GZGPU_INST(10)
GZGPU_INST(11)
GZGPU_INST(12)

}  // namespace gzgpu
