/*
 * gzoracle.c -- CPU oracle for the gzip decompression hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see gzoracle.h).  Never linked by the product.
 *
 * A plain-C restatement of the reference decode path (JackDanger/gzippy
 * v0.8.0, a Rust port of rapidgzip).  Paths below are relative to the
 * reference project root.  Parity is pinned by tests/test_oracle.py:
 *   - the 30 GZBLK01 known-answer blocks (corpus/silesia_blocks/NNN.bin),
 *   - system zlib 1.3 inflate on every generated input,
 *   - the block finder's branch-free scan against its own per-bit predicate.
 */
#define _GNU_SOURCE
#include "gzoracle.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* RFC 1951 constants (3.2.5, 3.2.6, 3.2.7).                                  */
/* ------------------------------------------------------------------------ */
static const uint16_t LEN_BASE[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,
                                      15, 17, 19, 23, 27, 31, 35, 43, 51,  59,
                                      67, 83, 99, 115, 131, 163, 195, 227, 258};
static const uint8_t LEN_EXTRA[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                      2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
static const uint16_t DIST_BASE[30] = {1,    2,    3,    4,    5,    7,     9,     13,
                                       17,   25,   33,   49,   65,   97,    129,   193,
                                       257,  385,  513,  769,  1025, 1537,  2049,  3073,
                                       4097, 6145, 8193, 12289, 16385, 24577};
static const uint8_t DIST_EXTRA[30] = {0, 0, 0, 0, 1, 1, 2, 2,  3,  3,  4,  4,  5,  5,  6,
                                       6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
static const uint8_t CL_ORDER[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

#define WIN 32768u
#define MARKER_BASE 32768u

/* ------------------------------------------------------------------------ */
/* CRC32 (reflected poly 0xEDB88320) and GF(2) combine.                        */
/* Follows src/decompress/parallel/crc32.rs:44-133 (polynomial_multiply_modulo */
/* :64, X2N table :90, x_power_modulo :104, combine_crc32 :127).              */
/* ------------------------------------------------------------------------ */
static uint32_t crc_tab[8][256];
static pthread_once_t crc_once = PTHREAD_ONCE_INIT;

static void crc_init(void) {
  for (uint32_t i = 0; i < 256; i++) {
    uint32_t c = i;
    for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
    crc_tab[0][i] = c;
  }
  for (int t = 1; t < 8; t++)
    for (uint32_t i = 0; i < 256; i++)
      crc_tab[t][i] = (crc_tab[t - 1][i] >> 8) ^ crc_tab[0][crc_tab[t - 1][i] & 0xFF];
}

uint32_t orc_crc32(uint32_t crc, const uint8_t *p, size_t n) {
  pthread_once(&crc_once, crc_init);
  uint32_t c = ~crc;
  while (n >= 8) {
    uint32_t lo, hi;
    memcpy(&lo, p, 4);
    memcpy(&hi, p + 4, 4);
    lo ^= c;
    c = crc_tab[7][lo & 0xFF] ^ crc_tab[6][(lo >> 8) & 0xFF] ^ crc_tab[5][(lo >> 16) & 0xFF] ^
        crc_tab[4][lo >> 24] ^ crc_tab[3][hi & 0xFF] ^ crc_tab[2][(hi >> 8) & 0xFF] ^
        crc_tab[1][(hi >> 16) & 0xFF] ^ crc_tab[0][hi >> 24];
    p += 8;
    n -= 8;
  }
  while (n--) c = (c >> 8) ^ crc_tab[0][(c ^ *p++) & 0xFF];
  return ~c;
}

/* a(x)*b(x) mod P(x), reflected bit order (bit 31 = x^0). */
uint32_t orc_gf2_mulmod(uint32_t a, uint32_t b) {
  uint32_t r = 0;
  for (uint32_t m = 1u << 31; m; m >>= 1) {
    if (a & m) r ^= b;
    b = (b & 1) ? (b >> 1) ^ 0xEDB88320u : b >> 1;
  }
  return r;
}

/* x^(8*nbytes) mod P, by square-and-multiply over x^(2^k). */
uint32_t orc_x_pow_8n(uint64_t nbytes) {
  static uint32_t x2n[32];
  static int init = 0;
  if (!init) {
    uint32_t v = 1u << 30; /* x^1 */
    for (int k = 0; k < 32; k++) {
      x2n[k] = v;
      v = orc_gf2_mulmod(v, v);
    }
    init = 1;
  }
  uint64_t e = nbytes * 8;
  uint32_t p = 1u << 31; /* x^0 */
  for (int k = 0; e; e >>= 1, k++)
    if (e & 1) p = orc_gf2_mulmod(x2n[k & 31], p);
  return p;
}

uint32_t orc_crc32_combine(uint32_t crc1, uint32_t crc2, uint64_t len2) {
  return orc_gf2_mulmod(orc_x_pow_8n(len2), crc1) ^ crc2;
}

/* ------------------------------------------------------------------------ */
/* gzip header (RFC 1952 2.3); follows src/decompress/parallel/gzip_format.rs */
/* read_header :47-133.                                                       */
/* ------------------------------------------------------------------------ */
int orc_gzip_header(const uint8_t *p, size_t n, size_t *hdr_len) {
  if (n < 10) return ORC_TRUNCATED;
  if (p[0] != 0x1f || p[1] != 0x8b || p[2] != 8) return ORC_BAD_HEADER;
  uint8_t flg = p[3];
  if (flg & 0xE0) return ORC_BAD_HEADER;
  size_t o = 10;
  if (flg & 4) {
    if (o + 2 > n) return ORC_TRUNCATED;
    size_t xlen = p[o] | (p[o + 1] << 8);
    o += 2;
    if (o + xlen > n) return ORC_TRUNCATED;
    o += xlen;
  }
  for (int f = 8; f <= 16; f <<= 1) { /* FNAME then FCOMMENT */
    if (flg & f) {
      while (o < n && p[o]) o++;
      if (o >= n) return ORC_TRUNCATED;
      o++;
    }
  }
  if (flg & 2) {
    if (o + 2 > n) return ORC_TRUNCATED;
    o += 2;
  }
  *hdr_len = o;
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Bit reader: LSB-first (src/decompress/parallel/bit_reader.rs).             */
/* Bytes past the end read as zero; `pos > 8*n` after a read = overrun.        */
/* ------------------------------------------------------------------------ */
typedef struct {
  const uint8_t *d;
  size_t n;
  uint64_t pos;
} br_t;

static inline uint64_t br_peek(const br_t *b, int k) { /* k <= 56 */
  size_t byte = (size_t)(b->pos >> 3);
  int sh = (int)(b->pos & 7);
  uint64_t v = 0;
  if (byte + 8 <= b->n) {
    memcpy(&v, b->d + byte, 8);
  } else {
    for (int i = 0; i < 8 && byte + i < b->n; i++) v |= (uint64_t)b->d[byte + i] << (8 * i);
  }
  return (v >> sh) & ((k >= 64) ? ~0ull : ((1ull << k) - 1));
}
static inline uint64_t br_read(br_t *b, int k) {
  uint64_t v = br_peek(b, k);
  b->pos += k;
  return v;
}
static inline int br_over(const br_t *b) { return b->pos > (uint64_t)b->n * 8; }

static uint64_t bits_at(const uint8_t *d, size_t n, uint64_t bit, int k) {
  br_t b = {d, n, bit};
  return br_peek(&b, k);
}

/* ------------------------------------------------------------------------ */
/* Canonical Huffman decoding tables: a PB-bit primary LUT of (sym, len) for   */
/* codes of at most PB bits; longer codes decode by the canonical first-code  */
/* search (RFC 1951 3.2.2).                                                   */
/* ------------------------------------------------------------------------ */
#define PB 10
typedef struct {
  uint32_t lut[1 << PB]; /* (sym << 4) | len ; len 0 = longer code or invalid */
  uint16_t count[16];
  uint16_t first[16];
  uint16_t offs[16];
  uint16_t sorted[320];
} htab_t;

static inline uint32_t rev_bits(uint32_t v, int n) {
  uint32_t r = 0;
  for (int i = 0; i < n; i++) {
    r = (r << 1) | (v & 1);
    v >>= 1;
  }
  return r;
}

/* zlib-compatible acceptance: over-subscribed sets are rejected; an
 * incomplete set is accepted only when its longest code has one bit (one
 * symbol) or it is empty. */
static int htab_build(htab_t *h, const uint8_t *lens, int nsym) {
  memset(h->count, 0, sizeof h->count);
  for (int s = 0; s < nsym; s++) h->count[lens[s]]++;
  h->count[0] = 0;
  int max = 15;
  while (max >= 1 && h->count[max] == 0) max--;
  int left = 1;
  for (int l = 1; l <= 15; l++) {
    left <<= 1;
    left -= h->count[l];
    if (left < 0) return -1;
  }
  if (max > 0 && left > 0 && max != 1) return -1;
  /* canonical first code per length: first[l] = (first[l-1] + count[l-1]) << 1 */
  uint32_t c = 0;
  uint16_t off = 0;
  h->first[0] = 0;
  for (int l = 1; l <= 15; l++) {
    c = l == 1 ? 0 : (c + h->count[l - 1]) << 1;
    h->first[l] = (uint16_t)c;
    h->offs[l] = off;
    off += h->count[l];
  }
  uint16_t next[16];
  memcpy(next, h->offs, sizeof next);
  for (int s = 0; s < nsym; s++)
    if (lens[s]) h->sorted[next[lens[s]]++] = (uint16_t)s;
  for (int i = 0; i < (1 << PB); i++) h->lut[i] = 0;
  for (int l = 1; l <= PB; l++) {
    for (int k = 0; k < h->count[l]; k++) {
      uint32_t s = h->sorted[h->offs[l] + k];
      uint32_t r = rev_bits(h->first[l] + k, l);
      for (uint32_t j = r; j < (1u << PB); j += 1u << l) h->lut[j] = (s << 4) | l;
    }
  }
  return 0;
}

/* returns symbol or -1 (invalid code) */
static inline int htab_decode(const htab_t *h, br_t *b) {
  uint32_t bits = (uint32_t)br_peek(b, 15);
  uint32_t e = h->lut[bits & ((1u << PB) - 1)];
  if (e & 15) {
    b->pos += e & 15;
    return (int)(e >> 4);
  }
  uint32_t c15 = rev_bits(bits, 15);
  for (int l = PB + 1; l <= 15; l++) {
    uint32_t code = c15 >> (15 - l);
    uint32_t idx = code - h->first[l];
    if (idx < h->count[l]) {
      b->pos += l;
      return h->sorted[h->offs[l] + idx];
    }
  }
  return -1;
}

static htab_t fixed_lit, fixed_dist;
static pthread_once_t fixed_once = PTHREAD_ONCE_INIT;
static void fixed_init(void) {
  uint8_t l[288];
  for (int i = 0; i < 144; i++) l[i] = 8;
  for (int i = 144; i < 256; i++) l[i] = 9;
  for (int i = 256; i < 280; i++) l[i] = 7;
  for (int i = 280; i < 288; i++) l[i] = 8;
  htab_build(&fixed_lit, l, 288);
  uint8_t d[32];
  for (int i = 0; i < 32; i++) d[i] = 5;
  htab_build(&fixed_dist, d, 32);
}

/* Dynamic block header (RFC 1951 3.2.7); the decoder counterpart of
 * src/decompress/parallel/marker_inflate.rs read_dynamic_huffman_coding
 * :1206.  Returns 0 or an ORC_* error. */
static int read_dynamic(br_t *b, htab_t *lit, htab_t *dist) {
  uint32_t h = (uint32_t)br_read(b, 14);
  int nlen = 257 + (h & 31), ndist = 1 + ((h >> 5) & 31), ncl = 4 + (h >> 10);
  if (nlen > 286 || ndist > 30) return ORC_BAD_DEFLATE;
  uint8_t cl[19] = {0};
  for (int i = 0; i < ncl; i++) cl[CL_ORDER[i]] = (uint8_t)br_read(b, 3);
  htab_t pre;
  if (htab_build(&pre, cl, 19) != 0) return ORC_BAD_DEFLATE;
  uint8_t lens[320];
  int i = 0;
  while (i < nlen + ndist) {
    int sym = htab_decode(&pre, b);
    if (sym < 0) return ORC_BAD_DEFLATE;
    if (sym < 16) {
      lens[i++] = (uint8_t)sym;
    } else {
      int rep;
      uint8_t v = 0;
      if (sym == 16) {
        if (i == 0) return ORC_BAD_DEFLATE;
        v = lens[i - 1];
        rep = 3 + (int)br_read(b, 2);
      } else if (sym == 17) {
        rep = 3 + (int)br_read(b, 3);
      } else {
        rep = 11 + (int)br_read(b, 7);
      }
      if (i + rep > nlen + ndist) return ORC_BAD_DEFLATE;
      while (rep--) lens[i++] = v;
    }
    if (br_over(b)) return ORC_TRUNCATED;
  }
  if (lens[256] == 0) return ORC_BAD_DEFLATE;
  if (htab_build(lit, lens, nlen) != 0) return ORC_BAD_DEFLATE;
  if (htab_build(dist, lens + nlen, ndist) != 0) return ORC_BAD_DEFLATE;
  return br_over(b) ? ORC_TRUNCATED : 0;
}

/* Parse a dynamic block header at `bit` and return its code lengths
 * (litlen then dist).  Used to pin the header parse against the GZBLK01
 * literal_cl / distance_cl fields. */
int orc_dynamic_lengths(const uint8_t *data, size_t n, uint64_t bit, uint8_t *lens, int *nlen,
                        int *ndist) {
  br_t b = {data, n, bit};
  uint32_t hdr = (uint32_t)br_read(&b, 3);
  if ((hdr >> 1) != 2) return ORC_BAD_DEFLATE;
  uint32_t h = (uint32_t)br_peek(&b, 14);
  *nlen = 257 + (h & 31);
  *ndist = 1 + ((h >> 5) & 31);
  htab_t *t = (htab_t *)malloc(2 * sizeof(htab_t));
  br_t b2 = b;
  int e = read_dynamic(&b2, &t[0], &t[1]);
  free(t);
  if (e) return e;
  /* re-read to recover the raw lengths */
  uint8_t cl[19] = {0};
  br_read(&b, 14);
  int ncl = 4 + (h >> 10);
  for (int i = 0; i < ncl; i++) cl[CL_ORDER[i]] = (uint8_t)br_read(&b, 3);
  htab_t pre;
  htab_build(&pre, cl, 19);
  int i = 0, total = *nlen + *ndist;
  while (i < total) {
    int sym = htab_decode(&pre, &b);
    if (sym < 16) {
      lens[i++] = (uint8_t)sym;
    } else {
      int rep;
      uint8_t v = 0;
      if (sym == 16) { v = lens[i - 1]; rep = 3 + (int)br_read(&b, 2); }
      else if (sym == 17) rep = 3 + (int)br_read(&b, 3);
      else rep = 11 + (int)br_read(&b, 7);
      while (rep--) lens[i++] = v;
    }
  }
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Chunk decode with u16 markers.                                             */
/* Marker semantics: src/decompress/parallel/marker_inflate.rs init_marker_zone */
/* :265 (a back-reference to window index w = 32768 + pos - dist emits        */
/* 32768 + w) and replace_markers.rs:7-23.  Stop rule: the first block         */
/* boundary >= stop_lo, as in chunk_decode.rs decode_chunk :225 with          */
/* stop_hint; the BFINAL block always ends the chunk.                          */
/* ------------------------------------------------------------------------ */
/* Core of orc_inflate_chunk, with the two modes of the device decoder's
 * sync starts (no counterpart in the reference):
 *   ORC_START_SYNC: start_bit is a symbol start inside the Huffman block
 *     whose header is at start_table (0: a non-final fixed-Huffman block);
 *   sync targets: the chunk's successors are sync starts t[0] < t[1] < ...;
 *     inside successor k's block (or a non-final fixed block, for a fixed
 *     sync start) the chunk stops at the symbol start == t[k]
 *     (*sync_end = 1).  Once it is past t[k], mid-block or at a block
 *     boundary, it has gone by successor k and moves on to k + 1; past the
 *     last one it stops only at the final block.
 * Without targets the stop rule is the first block boundary >= stop_lo. */
static int inflate_core(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t stop_lo,
                        int flags, uint64_t start_table, const uint64_t *targets,
                        const uint64_t *target_tables, size_t n_targets, int window_mode,
                        const uint8_t *window, size_t wlen, uint16_t *out, size_t cap,
                        orc_chunk_result *res, uint32_t *sync_end, uint64_t *end_hdr) {
  pthread_once(&fixed_once, fixed_init);
  br_t b = {data, n, start_bit};
  uint64_t o = 0, marker_end = 0;
  uint32_t nblocks = 0, nbt[3] = {0, 0, 0};
  int final_block = 0, st = ORC_OK, synced = 0;
  int in_sync = (flags & ORC_START_SYNC) != 0, tables_ready = 0;
  uint64_t blk_hdr = 0; /* header bit of the block being decoded (0 = unknown: a fixed sync start) */
  size_t cur = 0;
  htab_t *lit = NULL, *dist = NULL;
  htab_t *dyn = (htab_t *)malloc(2 * sizeof(htab_t));
  if (wlen > WIN) {
    window += wlen - WIN;
    wlen = WIN;
  }
  if (n_targets) stop_lo = targets[0];
  for (;;) {
    if (n_targets) {
      while (cur < n_targets && b.pos >= targets[cur]) cur++;
      stop_lo = cur < n_targets ? targets[cur] : (uint64_t)-1;
    }
    if (b.pos >= stop_lo) break;
    int bfinal, btype;
    tables_ready = 0;
    if (in_sync) {
      in_sync = 0;
      if (start_table) {
        /* the block's own header gives its type, BFINAL and code tables */
        br_t hb = {data, n, start_table};
        uint32_t hdr = (uint32_t)br_read(&hb, 3);
        bfinal = hdr & 1;
        btype = hdr >> 1;
        if (btype == 1) {
          lit = &fixed_lit;
          dist = &fixed_dist;
        } else if (btype == 2) {
          lit = &dyn[0];
          dist = &dyn[1];
          int e = read_dynamic(&hb, lit, dist);
          if (e) { st = e; break; }
        } else {
          st = ORC_BAD_DEFLATE;
          break;
        }
        tables_ready = 1;
        blk_hdr = start_table;
      } else {
        bfinal = 0;
        btype = 1;
        blk_hdr = 0;
      }
    } else {
      blk_hdr = b.pos;
      uint32_t hdr = (uint32_t)br_read(&b, 3);
      bfinal = hdr & 1;
      btype = hdr >> 1;
    }
    uint64_t watch = (uint64_t)-1;
    if (cur < n_targets) {
      const uint64_t tt = target_tables ? target_tables[cur] : 0;
      const int same = tt ? (blk_hdr == tt) : (btype == 1 && !bfinal);
      if (same) watch = targets[cur];
    }
    if (br_over(&b)) { st = ORC_TRUNCATED; break; }
    if (btype == 0) {
      b.pos = (b.pos + 7) & ~7ull;
      size_t byte = (size_t)(b.pos >> 3);
      if (byte + 4 > n) { st = ORC_TRUNCATED; break; }
      uint32_t len = data[byte] | (data[byte + 1] << 8);
      uint32_t nlen = data[byte + 2] | (data[byte + 3] << 8);
      if (len != (~nlen & 0xFFFFu)) { st = ORC_BAD_DEFLATE; break; }
      if (byte + 4 + len > n) { st = ORC_TRUNCATED; break; }
      if (o + len > cap) { st = ORC_OUT_TOO_SMALL; break; }
      for (uint32_t i = 0; i < len; i++) out[o++] = data[byte + 4 + i];
      b.pos += 8ull * (4 + len);
    } else if (btype == 1 || btype == 2) {
      if (tables_ready) {
        /* read from the block's header above */
      } else if (btype == 1) {
        lit = &fixed_lit;
        dist = &fixed_dist;
      } else {
        lit = &dyn[0];
        dist = &dyn[1];
        int e = read_dynamic(&b, lit, dist);
        if (e) { st = e; break; }
      }
      for (;;) {
        if (b.pos == watch) { synced = 1; break; }
        if (cur < n_targets && b.pos > targets[cur]) {
          /* went by a successor mid-block: a phantom; watch the next one */
          while (cur < n_targets && b.pos > targets[cur]) cur++;
          watch = (uint64_t)-1;
          if (cur < n_targets) {
            const uint64_t tt = target_tables ? target_tables[cur] : 0;
            if (tt ? (blk_hdr == tt) : (btype == 1 && !bfinal)) watch = targets[cur];
          }
        }
        if (br_over(&b)) { st = ORC_TRUNCATED; break; }
        int sym = htab_decode(lit, &b);
        if (sym < 0) { st = ORC_BAD_DEFLATE; break; }
        if (sym < 256) {
          if (o >= cap) { st = ORC_OUT_TOO_SMALL; break; }
          out[o++] = (uint16_t)sym;
          continue;
        }
        if (sym == 256) break;
        if (sym > 285) { st = ORC_BAD_DEFLATE; break; }
        uint32_t len = LEN_BASE[sym - 257] + (uint32_t)br_read(&b, LEN_EXTRA[sym - 257]);
        int ds = htab_decode(dist, &b);
        if (ds < 0 || ds >= 30) { st = ORC_BAD_DEFLATE; break; }
        uint32_t d = DIST_BASE[ds] + (uint32_t)br_read(&b, DIST_EXTRA[ds]);
        if (br_over(&b)) { st = ORC_TRUNCATED; break; }
        if (o + len > cap) { st = ORC_OUT_TOO_SMALL; break; }
        if ((uint64_t)d > o + WIN) { st = ORC_BAD_DEFLATE; break; }
        for (uint32_t j = 0; j < len; j++, o++) {
          int64_t s = (int64_t)o - (int64_t)d;
          uint16_t v;
          if (s >= 0) {
            v = out[s];
          } else {
            uint32_t w = (uint32_t)(WIN + s); /* window index, 0 = oldest */
            if (window_mode == ORC_WIN_MARKERS) {
              v = (uint16_t)(MARKER_BASE + w);
            } else {
              int64_t wi = (int64_t)w - (int64_t)(WIN - wlen);
              v = wi >= 0 ? window[wi] : 0;
            }
          }
          out[o] = v;
          if (v >= 256) marker_end = o + 1;
        }
      }
      if (st || synced) break;
      if (br_over(&b)) { st = ORC_TRUNCATED; break; }
    } else {
      st = ORC_BAD_DEFLATE;
      break;
    }
    nblocks++;
    nbt[btype]++;
    if (bfinal) {
      final_block = 1;
      break;
    }
  }
  free(dyn);
  if (sync_end) *sync_end = (uint32_t)synced;
  if (end_hdr) *end_hdr = synced ? blk_hdr : 0;
  res->end_bit = b.pos;
  res->out_len = o;
  res->marker_end = marker_end;
  res->n_blocks = nblocks;
  res->n_stored = nbt[0];
  res->n_fixed = nbt[1];
  res->n_dynamic = nbt[2];
  res->final_block = final_block;
  res->status = st;
  return st;
}

int orc_inflate_chunk(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t stop_lo,
                      int window_mode, const uint8_t *window, size_t wlen, uint16_t *out,
                      size_t cap, orc_chunk_result *res) {
  return inflate_core(data, n, start_bit, stop_lo, 0, 0, NULL, NULL, 0, window_mode, window, wlen,
                      out, cap, res, NULL, NULL);
}

int orc_inflate_chunk_ex(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t stop_lo,
                         int flags, uint64_t start_table, const uint64_t *sync_targets,
                         const uint64_t *target_tables, size_t n_targets, uint16_t *out,
                         size_t cap, orc_chunk_result *res, uint32_t *sync_end,
                         uint64_t *end_hdr) {
  return inflate_core(data, n, start_bit, stop_lo, flags, start_table, sync_targets, target_tables,
                      n_targets, (flags & ORC_ZERO_WINDOW) ? ORC_WIN_BYTES : ORC_WIN_MARKERS,
                      NULL, 0, out, cap, res, sync_end, end_hdr);
}

/* ------------------------------------------------------------------------ */
/* Sync starts in fixed-Huffman data (no counterpart in the reference; the  */
/* device finder's fixed_walk / sync search restated for the parity tests). */
/* ------------------------------------------------------------------------ */
static const uint8_t FW_LEN_EXTRA[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2,
                                         2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
static const uint8_t FW_DIST_EXTRA[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                          6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
#define SYNC_FAIL ((uint64_t)-1)

static uint64_t fixed_walk(const uint8_t *d, size_t n, uint64_t p, uint64_t target) {
  while (p < target) {
    uint32_t x = (uint32_t)bits_at(d, n, p, 9);
    uint32_t c7 = rev_bits(x & 127u, 7), c8 = rev_bits(x & 255u, 8), sym;
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
      sym = 144 + (rev_bits(x, 9) - 0x190);
      p += 9;
    }
    if (sym < 256) continue;
    if (sym == 256) {
      if ((bits_at(d, n, p, 3) >> 1) != 1) return SYNC_FAIL;
      p += 3;
      continue;
    }
    if (sym > 285) return SYNC_FAIL;
    p += FW_LEN_EXTRA[sym - 257];
    uint32_t dc = rev_bits((uint32_t)bits_at(d, n, p, 5), 5);
    if (dc >= 30) return SYNC_FAIL;
    p += 5 + FW_DIST_EXTRA[dc];
  }
  return p;
}

int orc_fixed_sync_find(const uint8_t *data, size_t n, uint64_t from, uint64_t to, uint64_t *bit) {
  const uint64_t target = from + ORC_SYNC_OFFSETS + ORC_SYNC_SPAN;
  if (target + 64 > to || target + 128 > (uint64_t)n * 8) return 0;
  uint64_t e[ORC_SYNC_OFFSETS];
  for (int i = 0; i < ORC_SYNC_OFFSETS; i++) e[i] = fixed_walk(data, n, from + i, target);
  uint64_t best = SYNC_FAIL;
  int best_n = 1;
  for (int i = 0; i < ORC_SYNC_OFFSETS; i++) {
    if (e[i] == SYNC_FAIL) continue;
    int c = 0;
    for (int j = 0; j < ORC_SYNC_OFFSETS; j++) c += e[j] == e[i];
    if (c > best_n || (c == best_n && best != SYNC_FAIL && e[i] < best)) {
      best = e[i];
      best_n = c;
    }
  }
  if (best == SYNC_FAIL) return 0;
  *bit = best;
  return 1;
}

/* Sync start inside the dynamic block whose header is at table_bit: the
 * positions of its code walked from ORC_SYNC_OFFSETS start bits of
 * [from, to) to the first symbol boundary >= from + offsets + span; an EOB
 * or an invalid code ends a walk as failed. */
int orc_dyn_sync_find(const uint8_t *data, size_t n, uint64_t table_bit, uint64_t from,
                      uint64_t to, uint64_t *bit) {
  const uint64_t target = from + ORC_SYNC_OFFSETS + ORC_SYNC_SPAN_DYN;
  if (target + 64 > to || target + 128 > (uint64_t)n * 8) return 0;
  br_t hb = {data, n, table_bit};
  if ((br_read(&hb, 3) >> 1) != 2) return 0;
  htab_t *t = (htab_t *)malloc(2 * sizeof(htab_t));
  if (read_dynamic(&hb, &t[0], &t[1])) {
    free(t);
    return 0;
  }
  uint64_t e[ORC_SYNC_OFFSETS];
  for (int i = 0; i < ORC_SYNC_OFFSETS; i++) {
    br_t b = {data, n, from + i};
    e[i] = SYNC_FAIL;
    while (b.pos < target) {
      int sym = htab_decode(&t[0], &b);
      if (sym < 0 || sym == 256 || sym > 285) break;
      if (sym > 256) {
        b.pos += LEN_EXTRA[sym - 257];
        int ds = htab_decode(&t[1], &b);
        if (ds < 0 || ds >= 30) break;
        b.pos += DIST_EXTRA[ds];
      }
      if (b.pos >= target) e[i] = b.pos;
    }
  }
  free(t);
  uint64_t best = SYNC_FAIL;
  int best_n = 1;
  for (int i = 0; i < ORC_SYNC_OFFSETS; i++) {
    if (e[i] == SYNC_FAIL) continue;
    int c = 0;
    for (int j = 0; j < ORC_SYNC_OFFSETS; j++) c += e[j] == e[i];
    if (c > best_n || (c == best_n && best != SYNC_FAIL && e[i] < best)) {
      best = e[i];
      best_n = c;
    }
  }
  if (best == SYNC_FAIL) return 0;
  *bit = best;
  return 1;
}

void orc_resolve_markers(const uint16_t *in, size_t n, const uint8_t *window32k, uint8_t *out) {
  for (size_t i = 0; i < n; i++) {
    uint16_t v = in[i];
    out[i] = v < 256 ? (uint8_t)v : window32k[v - MARKER_BASE];
  }
}

/* ------------------------------------------------------------------------ */
/* Block finder.                                                              */
/* Dynamic candidates follow src/decompress/parallel/blockfinder_validation.rs */
/* (skip LUT :68-150, validate_precode :190-226, find_dynamic_blocks_scalar    */
/* :631-750, parse_precode, is_valid_huffman_lengths :807-830,                */
/* validate_huffman_codes :836-925).  Stored candidates follow                */
/* find_uncompressed_blocks :370-475.  No fixed-Huffman candidates.           */
/* ------------------------------------------------------------------------ */
static int8_t skip_lut[1 << 15];
static pthread_once_t skip_once = PTHREAD_ONCE_INIT;

/* the 13-bit header filter, looking only at the `known` low bits */
static int hdr_filter(uint32_t bits, int known) {
  if (known == 0) return 0;
  int ok = !(bits & 1);
  if (known <= 1) return ok;
  uint32_t bt = (bits >> 1) & 3;
  ok &= (bt & 1) == 0;
  if (known <= 2) return ok;
  ok &= bt == 2;
  if (known < 8) return ok;
  ok &= ((bits >> 3) & 31) <= 29;
  if (known < 13) return ok;
  ok &= ((bits >> 8) & 31) <= 29;
  return ok;
}
static int next_cand(uint32_t bits, int known) {
  int s = 0;
  while (known > 0 && !hdr_filter(bits, known)) {
    bits >>= 1;
    known--;
    s++;
  }
  return s;
}
static void skip_init(void) {
  for (uint32_t i = 0; i < (1u << 15); i++) {
    int s = next_cand(i, 15);
    skip_lut[i] = (int8_t)(s == 0 ? 0 : s);
  }
}

/* Kraft equality over 15-bit leaves, or the one-code-of-length-1 tree. */
static int lengths_complete(const uint8_t *l, int n) {
  uint32_t leaves = 0, gt1 = 0;
  for (int i = 0; i < n; i++) {
    if (l[i] == 0) continue;
    if (l[i] > 15) return 0;
    leaves += 1u << (15 - l[i]);
    gt1 += l[i] > 1;
  }
  if (leaves == (1u << 14)) return gt1 == 0;
  return leaves == (1u << 15);
}

/* any_final: accept BFINAL = 1 too (the header of a block that follows a
 * stored candidate, stored_successor_ok) */
static int dyn_candidate_h(const uint8_t *data, size_t n, uint64_t bit, int any_final) {
  uint64_t nbits = (uint64_t)n * 8;
  if (bit + 17 > nbits) return 0;
  uint32_t h = (uint32_t)bits_at(data, n, bit, 17);
  if (!hdr_filter(any_final ? h & ~1u : h, 13)) return 0;
  int hlit = (h >> 3) & 31, hdist = (h >> 8) & 31, hclen = (h >> 13) & 15;
  int pc = hclen + 4;
  if (bit + 17 + 3 * pc > nbits) return 0;
  uint64_t pbits = bits_at(data, n, bit + 17, 3 * pc);
  /* validate_precode: leaf count over a depth-7 tree must be 128 or 64 */
  uint32_t leaves = 0;
  uint8_t cl[19] = {0};
  for (int i = 0; i < pc; i++) {
    uint32_t L = (pbits >> (3 * i)) & 7;
    if (L) leaves += 1u << (7 - L);
    cl[CL_ORDER[i]] = (uint8_t)L;
  }
  if (leaves != 128 && leaves != 64) return 0;
  if (!lengths_complete(cl, 19)) return 0;
  htab_t pre;
  if (htab_build(&pre, cl, 19) != 0) return 0;
  br_t b = {data, n, bit + 17 + 3 * pc};
  int hl = 257 + hlit, total = hl + 1 + hdist;
  uint8_t lens[320];
  int i = 0;
  while (i < total) {
    if (b.pos >= nbits) return 0;
    int sym = htab_decode(&pre, &b);
    if (sym < 0) return 0;
    if (sym < 16) {
      lens[i++] = (uint8_t)sym;
    } else {
      int rep;
      uint8_t v = 0;
      if (sym == 16) {
        if (i == 0) return 0;
        v = lens[i - 1];
        rep = 3 + (int)br_read(&b, 2);
      } else if (sym == 17) {
        rep = 3 + (int)br_read(&b, 3);
      } else {
        rep = 11 + (int)br_read(&b, 7);
      }
      if (i + rep > total) return 0;
      while (rep--) lens[i++] = v;
    }
    if (b.pos > nbits) return 0;
  }
  if (lens[256] == 0) return 0;
  return lengths_complete(lens, hl) && lengths_complete(lens + hl, total - hl);
}

static int dyn_candidate(const uint8_t *data, size_t n, uint64_t bit) {
  return dyn_candidate_h(data, n, bit, 0);
}

/* The block after a true non-final stored block starts at byte nb: another
 * stored block (LEN == ~NLEN one byte on) or a dynamic block passing the
 * full header predicate.  The device's partition-start rule (finder_core.cuh
 * stored_successor_ok), not the reference finder's: orc_find_blocks keeps
 * the reference predicate, orc_find_starts adds this. */
static int stored_successor_ok(const uint8_t *d, size_t n, uint64_t nb) {
  if (nb >= n) return 0;
  uint32_t bt = (d[nb] >> 1) & 3;
  if (bt == 0) {
    if (nb + 5 > n) return 0;
    uint32_t sz = d[nb + 1] | (d[nb + 2] << 8) | ((uint32_t)d[nb + 3] << 16) |
                  ((uint32_t)d[nb + 4] << 24);
    return ((sz ^ (sz >> 16)) & 0xFFFF) == 0xFFFF;
  }
  return bt == 2 && dyn_candidate_h(d, n, nb * 8, 1);
}

int orc_is_dynamic_candidate(const uint8_t *data, size_t n, uint64_t bit) {
  return dyn_candidate(data, n, bit);
}

typedef struct {
  uint64_t first, seek;
} cand_t;

static int cand_cmp(const void *a, const void *b) {
  const cand_t *x = a, *y = b;
  if (x->first != y->first) return x->first < y->first ? -1 : 1;
  if (x->seek != y->seek) return x->seek < y->seek ? -1 : 1;
  return 0;
}

static size_t find_stored(const uint8_t *d, size_t n, uint64_t start_bit, uint64_t end_bit,
                          cand_t *out, size_t cap, int succ) {
  size_t k = 0;
  if (n < 5) return 0;
  uint64_t until = (end_bit + 7) / 8;
  if (until > n - 4) until = n - 4;
  uint64_t sb = (start_bit + 3 + 7) / 8;
  if (sb < 2) sb = 2; /* need 10 preceding bits */
  for (uint64_t off = sb; off < until; off++) {
    uint32_t sz = d[off] | (d[off + 1] << 8) | ((uint32_t)d[off + 2] << 16) |
                  ((uint32_t)d[off + 3] << 24);
    if (((sz ^ (sz >> 16)) & 0xFFFF) != 0xFFFF) continue;
    uint64_t byte_bit = off * 8;
    uint32_t pre = (uint32_t)bits_at(d, n, byte_bit - 10, 10);
    if (pre & (7u << 7)) continue;
    int tz = 3;
    for (int j = 4; j <= 10; j++) {
      if (pre & (1u << (10 - j))) break;
      tz = j;
    }
    uint64_t earliest = byte_bit - tz, latest = byte_bit - 3;
    if (earliest >= start_bit && latest < end_bit) {
      uint32_t len = sz & 0xFFFF;
      if (len == 0 || off + 4 + len > n) continue;
      if (succ && !stored_successor_ok(d, n, off + 4 + len)) continue;
      if (k < cap) out[k] = (cand_t){earliest, latest};
      k++;
    }
  }
  return k;
}

static size_t find_blocks_impl(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t end_bit,
                               uint64_t *first, uint64_t *seek, size_t cap, int succ) {
  pthread_once(&skip_once, skip_init);
  uint64_t nbits = (uint64_t)n * 8;
  if (end_bit > nbits) end_bit = nbits;
  size_t k = 0, kcap = 64;
  cand_t *c = (cand_t *)malloc(kcap * sizeof(cand_t));
  uint64_t p = start_bit;
  while (p < end_bit) {
    uint32_t w = (uint32_t)bits_at(data, n, p, 15);
    int s = skip_lut[w];
    if (s > 0) {
      p += s;
      continue;
    }
    if (dyn_candidate(data, n, p)) {
      if (k == kcap) c = (cand_t *)realloc(c, (kcap *= 2) * sizeof(cand_t));
      c[k++] = (cand_t){p, p};
    }
    p++;
  }
  size_t ns = find_stored(data, n, start_bit, end_bit, NULL, 0, succ);
  if (ns) {
    c = (cand_t *)realloc(c, (k + ns + 1) * sizeof(cand_t));
    find_stored(data, n, start_bit, end_bit, c + k, ns, succ);
    k += ns;
  }
  qsort(c, k, sizeof(cand_t), cand_cmp);
  size_t w = k < cap ? k : cap;
  for (size_t i = 0; i < w; i++) {
    first[i] = c[i].first;
    seek[i] = c[i].seek;
  }
  free(c);
  return k;
}

size_t orc_find_blocks(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t end_bit,
                       uint64_t *first, uint64_t *seek, size_t cap) {
  return find_blocks_impl(data, n, start_bit, end_bit, first, seek, cap, 0);
}

size_t orc_find_starts(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t end_bit,
                       uint64_t *first, uint64_t *seek, size_t cap) {
  return find_blocks_impl(data, n, start_bit, end_bit, first, seek, cap, 1);
}

/* first stored candidate (in byte order, hence smallest bit_offset) */
static int find_stored_first(const uint8_t *d, size_t n, uint64_t start_bit, uint64_t end_bit,
                             cand_t *out) {
  if (n < 5) return 0;
  uint64_t until = (end_bit + 7) / 8;
  if (until > n - 4) until = n - 4;
  uint64_t sb = (start_bit + 3 + 7) / 8;
  if (sb < 2) sb = 2;
  for (uint64_t off = sb; off < until; off++) {
    uint32_t sz = d[off] | (d[off + 1] << 8) | ((uint32_t)d[off + 2] << 16) |
                  ((uint32_t)d[off + 3] << 24);
    if (((sz ^ (sz >> 16)) & 0xFFFF) != 0xFFFF) continue;
    cand_t c;
    if (find_stored(d, n, start_bit, end_bit < off * 8 + 1 ? end_bit : off * 8 + 1, &c, 1, 0) &&
        c.seek == off * 8 - 3) {
      *out = c;
      return 1;
    }
  }
  return 0;
}

/* The first candidate in (bit_offset, seek_bit) order among candidates with
 * bit_offset in [from, to): the start a speculative chunk decodes from
 * (blockfinder_validation.rs find_first_candidate :319-330).  0 if none. */
static int find_first(const uint8_t *data, size_t n, uint64_t from, uint64_t to, uint64_t *lo,
                      uint64_t *hi) {
  pthread_once(&skip_once, skip_init);
  uint64_t nbits = (uint64_t)n * 8;
  if (to > nbits) to = nbits;
  cand_t s;
  int have = find_stored_first(data, n, from, to, &s);
  uint64_t lim = have ? s.first + 1 : to; /* a dynamic tie at s.first sorts first */
  for (uint64_t p = from; p < lim;) {
    int k = skip_lut[(uint32_t)bits_at(data, n, p, 15)];
    if (k > 0) {
      p += k;
      continue;
    }
    if (dyn_candidate(data, n, p)) {
      *lo = *hi = p;
      return 1;
    }
    p++;
  }
  if (have) {
    *lo = s.first;
    *hi = s.seek;
  }
  return have;
}

/* ------------------------------------------------------------------------ */
/* Member scan: restates src/decompress/bgzf.rs scan_member_boundaries_fast    */
/* :2090-2230 and parse_gzip_header :2047.  Returns 0 for "not multi-member". */
/* ------------------------------------------------------------------------ */
static size_t scan_members(const uint8_t *d, size_t n, orc_member *out, size_t cap, int strict);

size_t orc_scan_members(const uint8_t *d, size_t n, orc_member *out, size_t cap) {
  return scan_members(d, n, out, cap, 0);
}

/* strict: also require the header plausibility of is_likely_multi_member
 * (src/decompress/format.rs:92-125: MTIME, XFL, OS), as the device scan does */
static size_t scan_members(const uint8_t *d, size_t n, orc_member *out, size_t cap, int strict) {
  if (n < 18 || d[0] != 0x1f || d[1] != 0x8b || d[2] != 8) return 0;
  size_t h0 = 10;
  if (orc_gzip_header(d, n, &h0) != ORC_OK) h0 = 10;
  size_t ns = 1, scap = 1024;
  uint64_t *starts = (uint64_t *)malloc(scap * sizeof(uint64_t));
  starts[0] = 0;
  size_t from = h0 + 1;
  while (from + 10 < n) {
    const uint8_t *hit = (const uint8_t *)memmem(d + from, n - from, "\x1f\x8b\x08", 3);
    if (!hit) break;
    size_t pos = (size_t)(hit - d);
    if (pos + 10 >= n) break;
    if ((d[pos + 3] & 0xE0) == 0 && pos >= 4) {
      uint32_t is = d[pos - 4] | (d[pos - 3] << 8) | ((uint32_t)d[pos - 2] << 16) |
                    ((uint32_t)d[pos - 1] << 24);
      uint32_t mt = d[pos + 4] | (d[pos + 5] << 8) | ((uint32_t)d[pos + 6] << 16) |
                    ((uint32_t)d[pos + 7] << 24);
      int plausible = mt <= 4102444800u && (d[pos + 8] == 0 || d[pos + 8] == 2 || d[pos + 8] == 4) &&
                      (d[pos + 9] <= 13 || d[pos + 9] == 255);
      if (is > 0 && is <= (1u << 30) && (!strict || plausible)) {
        if (ns == scap) starts = (uint64_t *)realloc(starts, (scap *= 2) * sizeof(uint64_t));
        starts[ns++] = pos;
      }
    }
    from = pos + 1;
  }
  size_t result = 0;
  if (ns >= 2) {
    uint64_t oo = 0;
    int ok = 1;
    for (size_t i = 0; i < ns && ok; i++) {
      uint64_t s = starts[i], e = i + 1 < ns ? starts[i + 1] : n;
      if (e - s < 18) { ok = 0; break; }
      uint32_t is = d[e - 4] | (d[e - 3] << 8) | ((uint32_t)d[e - 2] << 16) |
                    ((uint32_t)d[e - 1] << 24);
      /* parse_gzip_header(data, start, end) */
      uint64_t ds = s + 10;
      uint8_t flg = d[s + 3];
      if (flg & 4) {
        if (ds + 2 > e) { ok = 0; break; }
        ds += 2 + (d[ds] | (d[ds + 1] << 8));
      }
      if (flg & 8) { while (ds < e && d[ds]) ds++; ds++; }
      if (flg & 16) { while (ds < e && d[ds]) ds++; ds++; }
      if (flg & 2) ds += 2;
      if (ds >= e) { ok = 0; break; }
      if (i < cap) out[i] = (orc_member){s, e - s, ds, is, 0, oo};
      oo += is;
    }
    if (ok && oo <= (uint64_t)n * 100) result = ns;
  }
  free(starts);
  return result;
}

/* ------------------------------------------------------------------------ */
/* Whole-stream serial decode with the reference's stream semantics:           */
/* non-gzip -> NOT_GZIP (Ok(empty), src/lib.rs:50-52); members decoded in     */
/* order with CRC32 + ISIZE verified (src/decompress/mod.rs:742-870);         */
/* bytes after a member that do not start a gzip header end the walk cleanly. */
/* A back-reference before a member's first byte reads the zero window        */
/* (src/decompress/parallel/chunk_fetcher.rs:696).                            */
/* ------------------------------------------------------------------------ */
int orc_decompress(const uint8_t *in, size_t n, uint8_t *out, size_t cap, size_t *out_len) {
  *out_len = 0;
  if (n < 2 || in[0] != 0x1f || in[1] != 0x8b) return ORC_NOT_GZIP;
  size_t pos = 0, total = 0;
  int member = 0;
  while (pos < n) {
    if (member > 0) {
      if (n - pos < 18 || in[pos] != 0x1f || in[pos + 1] != 0x8b) break;
    }
    size_t hl;
    int hs = orc_gzip_header(in + pos, n - pos, &hl);
    if (hs != ORC_OK) {
      if (member == 0) return hs;
      break;
    }
    uint64_t sb = (uint64_t)(pos + hl) * 8;
    size_t tcap = (cap - total) + 1;
    uint16_t *tmp = (uint16_t *)malloc(tcap * sizeof(uint16_t));
    orc_chunk_result r;
    int st = orc_inflate_chunk(in, n, sb, ~0ull, ORC_WIN_BYTES, NULL, 0, tmp, tcap, &r);
    if (st == ORC_OUT_TOO_SMALL || (st == ORC_OK && r.out_len > cap - total)) {
      free(tmp);
      return ORC_OUT_TOO_SMALL;
    }
    if (st != ORC_OK) {
      free(tmp);
      return st;
    }
    if (!r.final_block) {
      free(tmp);
      return ORC_TRUNCATED;
    }
    for (uint64_t i = 0; i < r.out_len; i++) out[total + i] = (uint8_t)tmp[i];
    free(tmp);
    size_t tr = (size_t)((r.end_bit + 7) / 8);
    if (tr + 8 > n) return ORC_TRUNCATED;
    uint32_t crc = in[tr] | (in[tr + 1] << 8) | ((uint32_t)in[tr + 2] << 16) |
                   ((uint32_t)in[tr + 3] << 24);
    uint32_t isz = in[tr + 4] | (in[tr + 5] << 8) | ((uint32_t)in[tr + 6] << 16) |
                   ((uint32_t)in[tr + 7] << 24);
    if ((uint32_t)r.out_len != isz) return ORC_SIZE_MISMATCH;
    if (orc_crc32(0, out + total, r.out_len) != crc) return ORC_CRC_MISMATCH;
    total += r.out_len;
    *out_len = total;
    pos = tr + 8;
    member++;
  }
  *out_len = total;
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Chunked speculative decode (restates the single-member parallel driver:     */
/* src/decompress/parallel/chunk_fetcher.rs drive_impl :638-850, the chunk    */
/* protocol of consumer_loop :855 / try_speculative_decode_candidate          */
/* :2506-2595, and post-processing resolve_chunk_markers_on_chunk :1969 +     */
/* CRC combine in drain_one_pending :2944-3006).                              */
/*                                                                            */
/* Phases, mirroring the CUDA pipeline:                                       */
/*   1. partition each member's deflate range into chunk_bytes partitions;    */
/*      partition i>0 starts at the first finder candidate >= its guess;      */
/*   2. decode every chunk in parallel (first chunk of a member with the      */
/*      zero window, the rest window-absent with markers), stopping at the    */
/*      next chunk's start;                                                   */
/*   3. chain walk: a chunk is accepted when its predecessor's end bit lies in */
/*      its [first, seek] range; otherwise it is discarded and the gap is     */
/*      re-decoded from the predecessor's end (a confirmed boundary);         */
/*   4. prefix offsets; resolve every chunk's last 32 KiB in chain order;     */
/*      resolve the remaining entries in parallel;                            */
/*   5. per-chunk CRC in parallel, combined in order per member; verify       */
/*      CRC32 + ISIZE against each trailer.                                   */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint64_t lo, hi;     /* acceptable start range (first, seek) */
  uint64_t stop;       /* stop_lo */
  int member_first;    /* starts a member: zero window, no markers */
  int valid;           /* finder produced a start */
  int member;          /* member index */
  uint16_t *buf;
  size_t cap;
  orc_chunk_result r;
  uint64_t out_off;
  uint32_t crc;
} ochunk_t;

typedef struct {
  void (*fn)(void *, size_t);
  void *ctx;
  size_t n;
  atomic_size_t next;
} pfor_t;

static void *pfor_worker(void *a) {
  pfor_t *p = (pfor_t *)a;
  for (;;) {
    size_t i = atomic_fetch_add(&p->next, 1);
    if (i >= p->n) break;
    p->fn(p->ctx, i);
  }
  return NULL;
}

static void pfor(int threads, size_t n, void (*fn)(void *, size_t), void *ctx) {
  pfor_t p;
  p.fn = fn;
  p.ctx = ctx;
  p.n = n;
  atomic_init(&p.next, 0);
  if (threads <= 1 || n <= 1) {
    pfor_worker(&p);
    return;
  }
  pthread_t th[256];
  int t = threads > 256 ? 256 : threads;
  for (int i = 0; i < t; i++) pthread_create(&th[i], NULL, pfor_worker, &p);
  for (int i = 0; i < t; i++) pthread_join(th[i], NULL);
}

typedef struct {
  const uint8_t *in;
  size_t n;
  ochunk_t *c;
  uint64_t chunk_bits;
  uint64_t *guess;
  uint64_t *limit;
  uint8_t *out;
} cctx_t;

static void do_find(void *a, size_t i) {
  cctx_t *x = (cctx_t *)a;
  ochunk_t *c = &x->c[i];
  if (c->member_first) {
    c->valid = 1;
    return;
  }
  uint64_t lo, hi;
  c->valid = find_first(x->in, x->n, x->guess[i], x->limit[i], &lo, &hi);
  if (c->valid) {
    c->lo = lo;
    c->hi = hi;
  }
}

static void decode_one(const uint8_t *in, size_t n, ochunk_t *c, uint64_t start) {
  size_t cap = c->cap ? c->cap : 1 << 16;
  for (;;) {
    c->buf = (uint16_t *)realloc(c->buf, cap * sizeof(uint16_t));
    int st = orc_inflate_chunk(in, n, start, c->stop,
                               c->member_first ? ORC_WIN_BYTES : ORC_WIN_MARKERS, NULL, 0,
                               c->buf, cap, &c->r);
    if (st != ORC_OUT_TOO_SMALL || cap >= ((size_t)1 << 36)) break;
    cap *= 4;
  }
  c->cap = cap;
}

/* A failed speculative start moves on to the next candidate of the same
 * partition, up to 4 starts (speculative_decode_find_boundary,
 * chunk_fetcher.rs:2616-2740, tries the candidates in order). */
static void do_decode(void *a, size_t i) {
  cctx_t *x = (cctx_t *)a;
  ochunk_t *c = &x->c[i];
  if (!c->valid) return;
  for (int tries = 0;; tries++) {
    decode_one(x->in, x->n, c, c->hi);
    if (c->r.status == ORC_OK || c->member_first || tries + 1 >= 4) break;
    uint64_t lo, hi;
    if (!find_first(x->in, x->n, c->lo + 1, x->limit[i], &lo, &hi)) break;
    c->lo = lo;
    c->hi = hi;
  }
}

typedef struct {
  cctx_t *x;
  ochunk_t **order;
} rctx_t;

static void do_resolve_body(void *a, size_t k) {
  rctx_t *r = (rctx_t *)a;
  ochunk_t *c = r->order[k];
  uint8_t *out = r->x->out;
  uint64_t len = c->r.out_len, tail = len < WIN ? len : WIN;
  for (uint64_t i = 0; i < len - tail; i++) {
    uint16_t v = c->buf[i];
    if (v < 256) {
      out[c->out_off + i] = (uint8_t)v;
    } else {
      int64_t src = (int64_t)c->out_off - WIN + (v - MARKER_BASE);
      out[c->out_off + i] = src >= 0 ? out[src] : 0;
    }
  }
}

static void do_crc(void *a, size_t k) {
  rctx_t *r = (rctx_t *)a;
  ochunk_t *c = r->order[k];
  c->crc = orc_crc32(0, r->x->out + c->out_off, c->r.out_len);
}

int orc_decompress_chunked(const uint8_t *in, size_t n, size_t chunk_bytes, int threads,
                           uint8_t *out, size_t cap, size_t *out_len, orc_chunked_stats *st) {
  orc_chunked_stats dummy;
  if (!st) st = &dummy;
  memset(st, 0, sizeof *st);
  *out_len = 0;
  if (n < 2 || in[0] != 0x1f || in[1] != 0x8b) return ORC_NOT_GZIP;
  if (chunk_bytes < 4096) chunk_bytes = 4096;
  uint64_t cbits = (uint64_t)chunk_bytes * 8;

  /* member ranges: scan candidates, else one member spanning the input */
  size_t nm = scan_members(in, n, NULL, 0, 1);
  orc_member *mem = NULL;
  if (nm >= 2) {
    mem = (orc_member *)malloc(nm * sizeof(orc_member));
    scan_members(in, n, mem, nm, 1);
  } else {
    size_t hl;
    int hs = orc_gzip_header(in, n, &hl);
    if (hs != ORC_OK) return hs;
    nm = 1;
    mem = (orc_member *)malloc(sizeof(orc_member));
    mem[0] = (orc_member){0, n, hl, 0, 0, 0};
  }
  /* partition grid */
  size_t nc = 0, ccap = 1024;
  ochunk_t *ch = (ochunk_t *)calloc(ccap, sizeof(ochunk_t));
  uint64_t *guess = (uint64_t *)malloc(ccap * sizeof(uint64_t));
  uint64_t *limit = (uint64_t *)malloc(ccap * sizeof(uint64_t));
  for (size_t m = 0; m < nm; m++) {
    uint64_t b0 = mem[m].deflate_start * 8;
    uint64_t bend = (mem[m].start + mem[m].length) * 8;
    for (uint64_t g = b0; g < bend; g += cbits) {
      if (nc == ccap) {
        ccap *= 2;
        ch = (ochunk_t *)realloc(ch, ccap * sizeof(ochunk_t));
        guess = (uint64_t *)realloc(guess, ccap * sizeof(uint64_t));
        limit = (uint64_t *)realloc(limit, ccap * sizeof(uint64_t));
      }
      memset(&ch[nc], 0, sizeof(ochunk_t));
      ch[nc].member = (int)m;
      ch[nc].member_first = g == b0;
      ch[nc].lo = ch[nc].hi = g;
      guess[nc] = g;
      limit[nc] = g + cbits < bend ? g + cbits : bend;
      ch[nc].cap = (size_t)chunk_bytes * 4 + 65536;
      nc++;
    }
  }
  st->n_chunks = nc;
  st->n_members = nm;
  cctx_t x = {in, n, ch, cbits, guess, limit, out};
  pfor(threads, nc, do_find, &x);
  /* stop of each valid chunk = next valid chunk's lo */
  for (size_t i = 0; i < nc; i++) {
    if (!ch[i].valid) continue;
    st->n_candidates_ok++;
    ch[i].stop = ~0ull;
    for (size_t j = i + 1; j < nc; j++)
      if (ch[j].valid) {
        /* a member candidate ends its predecessor at its header bit: a real
         * one follows the BFINAL block, a false one lies inside the member */
        ch[i].stop = ch[j].member_first ? mem[ch[j].member].start * 8 : ch[j].lo;
        break;
      }
  }
  pfor(threads, nc, do_decode, &x);

  /* chain walk (consumer_loop semantics): accept a speculative chunk when the
   * confirmed end of its predecessor lies in its [lo, hi] start range, else
   * discard it and re-decode from the confirmed boundary. */
  int status = ORC_OK;
  size_t ocap = nc + 16, no = 0, nextra = 0, xcap = nc + 16;
  ochunk_t **order = (ochunk_t **)malloc(ocap * sizeof(ochunk_t *));
  ochunk_t **extra = (ochunk_t **)malloc(xcap * sizeof(ochunk_t *));
#define PUSH_ORDER(c)                                                              \
  do {                                                                             \
    if (no == ocap) order = (ochunk_t **)realloc(order, (ocap *= 2) * sizeof(ochunk_t *)); \
    order[no++] = (c);                                                             \
  } while (0)
#define NEW_REPAIR(var, start, stopv, mfirst)                                       \
  do {                                                                             \
    var = (ochunk_t *)calloc(1, sizeof(ochunk_t));                                 \
    var->valid = 1;                                                                \
    var->member_first = (mfirst);                                                  \
    var->lo = var->hi = (start);                                                   \
    var->stop = (stopv);                                                           \
    var->cap = (size_t)chunk_bytes * 4 + 65536;                                    \
    decode_one(in, n, var, (start));                                               \
    st->n_repairs++;                                                               \
    if (nextra == xcap) extra = (ochunk_t **)realloc(extra, (xcap *= 2) * sizeof(ochunk_t *)); \
    extra[nextra++] = var;                                                         \
  } while (0)
  uint64_t mpos = 0; /* byte offset of the next member header */
  size_t k0 = 0;
  for (int member = 0; status == ORC_OK; member++) {
    if (member > 0 && mpos >= n) break;
    ochunk_t *cur = NULL;
    size_t j = k0;
    while (j < nc && !(ch[j].valid && ch[j].member_first && mem[ch[j].member].start >= mpos)) j++;
    if (j < nc && mem[ch[j].member].start == mpos) {
      cur = &ch[j++];
    } else {
      size_t hl;
      if (member == 0) { status = ORC_BAD_HEADER; break; }
      if (n - mpos < 18 || in[mpos] != 0x1f || in[mpos + 1] != 0x8b ||
          orc_gzip_header(in + mpos, n - mpos, &hl) != ORC_OK)
        break; /* trailing bytes that start no member: stop cleanly */
      while (j < nc && !ch[j].valid) j++;
      NEW_REPAIR(cur, (uint64_t)(mpos + hl) * 8, ~0ull, 1);
    }
    for (;;) {
      PUSH_ORDER(cur);
      if (cur->r.status != ORC_OK) {
        status = cur->r.status == ORC_OUT_TOO_SMALL ? ORC_BAD_DEFLATE : cur->r.status;
        break;
      }
      if (cur->r.final_block) break;
      uint64_t e = cur->r.end_bit;
#define FIRST_BIT(k) (ch[k].member_first ? mem[ch[k].member].start * 8 : ch[k].lo)
      int accepted = 0;
      while (j < nc) {
        if (!ch[j].valid) { j++; continue; }
        if (!ch[j].member_first && e >= ch[j].lo && e <= ch[j].hi && ch[j].r.status == ORC_OK) {
          accepted = 1;
          break;
        }
        if (FIRST_BIT(j) > e) break;
        st->n_spec_rejected++;
        j++;
      }
      if (accepted) {
        cur = &ch[j++];
        continue;
      }
      if (cur->r.out_len == 0 && cur->r.n_blocks == 0 && cur->lo == e && cur != &ch[j - 1]) {
        status = ORC_BAD_DEFLATE; /* no progress */
        break;
      }
      uint64_t stop = j < nc ? FIRST_BIT(j) : ~0ull;
#undef FIRST_BIT
      ochunk_t *rep;
      NEW_REPAIR(rep, e, stop, 0);
      cur = rep;
    }
    if (status != ORC_OK) break;
    mpos = (cur->r.end_bit + 7) / 8 + 8;
    if (mpos > n) { status = ORC_TRUNCATED; break; }
    k0 = j;
  }
#undef PUSH_ORDER
#undef NEW_REPAIR

  /* prefix offsets + member segmentation (a member-first chunk opens one) */
  uint64_t total = 0;
  for (size_t k = 0; k < no; k++) {
    order[k]->out_off = total;
    total += order[k]->r.out_len;
  }
  if (status == ORC_OK && total > cap) status = ORC_OUT_TOO_SMALL;
  if (status == ORC_OK) {
    /* window chain: tails in order */
    for (size_t k = 0; k < no; k++) {
      ochunk_t *c = order[k];
      uint64_t len = c->r.out_len, t0 = len > WIN ? len - WIN : 0;
      if (c->r.marker_end > t0) st->n_tail_marker_chunks++;
      for (uint64_t q = t0; q < len; q++) {
        uint16_t v = c->buf[q];
        if (v < 256) {
          out[c->out_off + q] = (uint8_t)v;
        } else {
          int64_t src = (int64_t)c->out_off - WIN + (v - MARKER_BASE);
          out[c->out_off + q] = src >= 0 ? out[src] : 0;
        }
      }
    }
    rctx_t rc = {&x, order};
    pfor(threads, no, do_resolve_body, &rc);
    pfor(threads, no, do_crc, &rc);
    /* verify each member: a member-first chunk opens it, the BFINAL chunk closes it */
    uint32_t crc = 0;
    uint64_t mlen = 0;
    for (size_t k = 0; k < no && status == ORC_OK; k++) {
      ochunk_t *c = order[k];
      if (c->member_first) {
        crc = 0;
        mlen = 0;
      }
      crc = orc_crc32_combine(crc, c->crc, c->r.out_len);
      mlen += c->r.out_len;
      if (c->r.final_block) {
        size_t tr = (size_t)((c->r.end_bit + 7) / 8);
        uint32_t ecrc = in[tr] | (in[tr + 1] << 8) | ((uint32_t)in[tr + 2] << 16) |
                        ((uint32_t)in[tr + 3] << 24);
        uint32_t eisz = in[tr + 4] | (in[tr + 5] << 8) | ((uint32_t)in[tr + 6] << 16) |
                        ((uint32_t)in[tr + 7] << 24);
        if ((uint32_t)mlen != eisz) status = ORC_SIZE_MISMATCH;
        else if (crc != ecrc) status = ORC_CRC_MISMATCH;
      }
    }
    if (status == ORC_OK && no > 0 && !order[no - 1]->r.final_block) status = ORC_TRUNCATED;
  }
  *out_len = status == ORC_OK ? total : 0;
  for (size_t k = 0; k < nc; k++) free(ch[k].buf);
  for (size_t k = 0; k < nextra; k++) {
    free(extra[k]->buf);
    free(extra[k]);
  }
  free(extra);
  free(order);
  free(ch);
  free(guess);
  free(limit);
  free(mem);
  return status;
}
