/*
 * synth.c -- seeded synthetic inputs for the decompression workloads.
 *
 * Content types (4 MiB segments or whole members):
 *   0 MARKOV : order-2 Markov text over 96 printable ASCII symbols
 *              (0x20..0x7e plus '\n'), Zipf(1.1)-weighted transitions,
 *              interleaved with copies of earlier 8..256-byte spans at
 *              distances uniform in 1..32768 covering ~60% of the output;
 *   1 RANDOM : uniform random bytes (deflate emits stored blocks);
 *   2 RUNS   : runs of one random byte value, geometric length, mean 40;
 *   3 RAMPS  : uint16 little-endian ramps plus Gaussian noise, sigma = 8.
 *
 * Compression stands in for the reference's encoder with zlib
 * (deflateInit2(level, Z_DEFLATED, 31, 8, strategy)): levels 6 and 9 use
 * Z_DEFAULT_STRATEGY (dynamic blocks, stored for incompressible data) and
 * level 1 uses Z_FIXED, so level-1 members are fixed-Huffman as the
 * workload definition requires.  Every member is one serial deflate stream
 * (syn_gzip) unless a caller asks for the pigz-style framing
 * (syn_gzip_parallel): blocks compressed in parallel, each primed with the
 * previous 32 KiB as its dictionary and closed with Z_SYNC_FLUSH, then
 * framed as ONE gzip member.  Each Z_SYNC_FLUSH leaves a byte-aligned empty
 * stored block in the stream, a free block boundary a serial encoder would
 * not write, so that framing is kept only as a separately named workload.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

typedef struct {
  uint64_t s[4];
} rng_t;

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t splitmix(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static void rng_seed(rng_t *r, uint64_t seed) {
  for (int i = 0; i < 4; i++) r->s[i] = splitmix(&seed);
}
static inline uint64_t rng_next(rng_t *r) { /* xoshiro256** */
  uint64_t *s = r->s;
  uint64_t res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return res;
}
static inline double rng_unit(rng_t *r) { return (rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline uint64_t rng_below(rng_t *r, uint64_t n) { return (uint64_t)(rng_unit(r) * n); }
static inline uint64_t rng_geom(rng_t *r, double mean) { /* support 1.., mean `mean` */
  double p = 1.0 / mean, u = rng_unit(r);
  if (u <= 0) u = 1e-300;
  return 1 + (uint64_t)floor(log(u) / log(1.0 - p));
}

static const int NSYM = 96;
static inline uint8_t sym_char(int s) { return s == 95 ? '\n' : (uint8_t)(0x20 + s); }
static inline int char_sym(uint8_t c) { return c == '\n' ? 95 : (c >= 0x20 && c < 0x7f ? c - 0x20 : 0); }

static void gen_markov(rng_t *r, uint8_t *out, size_t n) {
  /* Zipf(1.1) rank CDF shared by every context; each context permutes the
   * symbols so its most likely successor differs. */
  double cdf[96], acc = 0;
  for (int k = 0; k < NSYM; k++) acc += 1.0 / pow(k + 1, 1.1);
  double run = 0;
  for (int k = 0; k < NSYM; k++) {
    run += 1.0 / pow(k + 1, 1.1) / acc;
    cdf[k] = run;
  }
  uint8_t *perm = (uint8_t *)malloc((size_t)NSYM * NSYM * NSYM);
  for (int c = 0; c < NSYM * NSYM; c++) {
    uint8_t *p = perm + (size_t)c * NSYM;
    for (int k = 0; k < NSYM; k++) p[k] = (uint8_t)k;
    for (int k = NSYM - 1; k > 0; k--) {
      int j = (int)rng_below(r, k + 1);
      uint8_t t = p[k];
      p[k] = p[j];
      p[j] = t;
    }
  }
  size_t o = 0;
  int c1 = 0, c2 = 0;
  while (o < n) {
    /* Markov run (mean 88 bytes) then a copy (8..256 bytes, mean 132): ~60% copied */
    size_t m = rng_geom(r, 88.0);
    for (size_t i = 0; i < m && o < n; i++) {
      double u = rng_unit(r);
      int lo = 0, hi = NSYM - 1;
      while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (cdf[mid] < u) lo = mid + 1; else hi = mid;
      }
      int s = perm[((size_t)c1 * NSYM + c2) * NSYM + lo];
      out[o++] = sym_char(s);
      c1 = c2;
      c2 = s;
    }
    if (o >= 16 && o < n) {
      size_t len = 8 + rng_below(r, 249);
      size_t maxd = o < 32768 ? o : 32768;
      size_t d = 1 + rng_below(r, maxd);
      for (size_t i = 0; i < len && o < n; i++, o++) out[o] = out[o - d];
      c1 = char_sym(out[o - 2]);
      c2 = char_sym(out[o - 1]);
    }
  }
  free(perm);
}

static void gen_random(rng_t *r, uint8_t *out, size_t n) {
  size_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t v = rng_next(r);
    memcpy(out + i, &v, 8);
  }
  for (; i < n; i++) out[i] = (uint8_t)rng_next(r);
}

static void gen_runs(rng_t *r, uint8_t *out, size_t n) {
  size_t o = 0;
  while (o < n) {
    uint8_t v = (uint8_t)rng_next(r);
    size_t len = rng_geom(r, 40.0);
    for (size_t i = 0; i < len && o < n; i++) out[o++] = v;
  }
}

static void gen_ramps(rng_t *r, uint8_t *out, size_t n) {
  size_t o = 0;
  while (o < n) {
    size_t len = 256 + rng_below(r, 3841);
    double v = (double)rng_below(r, 65536);
    double slope = (rng_unit(r) * 2.0 - 1.0) * 64.0;
    for (size_t i = 0; i < len && o < n; i++) {
      double u1 = rng_unit(r), u2 = rng_unit(r);
      if (u1 < 1e-300) u1 = 1e-300;
      double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2) * 8.0;
      long x = lround(v + g);
      uint16_t w = (uint16_t)(x & 0xFFFF);
      out[o++] = (uint8_t)(w & 0xFF);
      if (o < n) out[o++] = (uint8_t)(w >> 8);
      v += slope;
      if (v < 0) v += 65536;
      if (v >= 65536) v -= 65536;
    }
  }
}

void syn_content(int type, uint64_t seed, uint8_t *out, size_t n) {
  rng_t r;
  rng_seed(&r, seed * 0x2545F4914F6CDD1Dull + (uint64_t)type);
  switch (type) {
    case 0: gen_markov(&r, out, n); break;
    case 1: gen_random(&r, out, n); break;
    case 2: gen_runs(&r, out, n); break;
    default: gen_ramps(&r, out, n); break;
  }
}

/* ---------------------------------------------------------------------- */
/* gzip framing                                                           */
/* ---------------------------------------------------------------------- */
static int strategy_for(int level) { return level <= 1 ? Z_FIXED : Z_DEFAULT_STRATEGY; }

/* one member, serial zlib; returns compressed size or 0 on failure */
size_t syn_gzip(const uint8_t *in, size_t n, int level, uint8_t *out, size_t cap) {
  z_stream z;
  memset(&z, 0, sizeof z);
  if (deflateInit2(&z, level, Z_DEFLATED, 31, 8, strategy_for(level)) != Z_OK) return 0;
  z.next_in = (Bytef *)in;
  z.next_out = out;
  z.avail_out = 0;
  size_t left_in = n;
  size_t total_out = 0;
  int rc;
  do {
    uInt chunk_in = left_in > (1u << 30) ? (1u << 30) : (uInt)left_in;
    z.avail_in = chunk_in;
    left_in -= chunk_in;
    int flush = left_in ? Z_NO_FLUSH : Z_FINISH;
    do {
      size_t room = cap - total_out;
      z.avail_out = room > (1u << 30) ? (1u << 30) : (uInt)room;
      z.next_out = out + total_out;
      uInt before = z.avail_out;
      rc = deflate(&z, flush);
      total_out += before - z.avail_out;
      if (rc == Z_STREAM_ERROR || (z.avail_out == 0 && total_out == cap)) {
        deflateEnd(&z);
        return 0;
      }
    } while (z.avail_out == 0);
  } while (left_in);
  deflateEnd(&z);
  return rc == Z_STREAM_END ? total_out : 0;
}

typedef struct {
  const uint8_t *in;
  size_t n, block;
  int level;
  size_t nblocks;
  uint8_t **bout;
  size_t *blen;
  uint32_t *bcrc;
  size_t next;
  pthread_mutex_t mu;
} par_t;

static void *par_worker(void *a) {
  par_t *p = (par_t *)a;
  for (;;) {
    pthread_mutex_lock(&p->mu);
    size_t i = p->next++;
    pthread_mutex_unlock(&p->mu);
    if (i >= p->nblocks) break;
    size_t off = i * p->block, len = p->n - off < p->block ? p->n - off : p->block;
    z_stream z;
    memset(&z, 0, sizeof z);
    deflateInit2(&z, p->level, Z_DEFLATED, -15, 8, strategy_for(p->level));
    if (i > 0) {
      size_t d = off < 32768 ? off : 32768;
      deflateSetDictionary(&z, p->in + off - d, (uInt)d);
    }
    size_t cap = deflateBound(&z, len) + 64;
    uint8_t *o = (uint8_t *)malloc(cap);
    z.next_in = (Bytef *)(p->in + off);
    z.avail_in = (uInt)len;
    z.next_out = o;
    z.avail_out = (uInt)cap;
    deflate(&z, i + 1 == p->nblocks ? Z_FINISH : Z_SYNC_FLUSH);
    p->blen[i] = cap - z.avail_out;
    p->bout[i] = o;
    p->bcrc[i] = (uint32_t)crc32(0, p->in + off, (uInt)len);
    deflateEnd(&z);
  }
  return NULL;
}

/* one member compressed by `threads` workers in `block`-byte pieces */
size_t syn_gzip_parallel(const uint8_t *in, size_t n, int level, int threads, size_t block,
                         uint8_t *out, size_t cap) {
  if (block < 65536) block = 65536;
  par_t p;
  memset(&p, 0, sizeof p);
  p.in = in;
  p.n = n;
  p.block = block;
  p.level = level;
  p.nblocks = n ? (n + block - 1) / block : 1;
  p.bout = (uint8_t **)calloc(p.nblocks, sizeof(uint8_t *));
  p.blen = (size_t *)calloc(p.nblocks, sizeof(size_t));
  p.bcrc = (uint32_t *)calloc(p.nblocks, sizeof(uint32_t));
  pthread_mutex_init(&p.mu, NULL);
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t th[256];
  for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, par_worker, &p);
  for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
  size_t o = 0, ok = 1;
  static const uint8_t hdr[10] = {0x1f, 0x8b, 8, 0, 0, 0, 0, 0, 0, 3};
  if (cap < 18) ok = 0;
  if (ok) {
    memcpy(out, hdr, 10);
    o = 10;
  }
  uint32_t crc = 0;
  for (size_t i = 0; i < p.nblocks; i++) {
    if (ok && o + p.blen[i] + 8 <= cap) {
      memcpy(out + o, p.bout[i], p.blen[i]);
      o += p.blen[i];
    } else {
      ok = 0;
    }
    size_t len = (i + 1 == p.nblocks) ? n - i * block : block;
    crc = i == 0 ? p.bcrc[0] : (uint32_t)crc32_combine(crc, p.bcrc[i], (z_off_t)len);
    free(p.bout[i]);
  }
  if (ok) {
    for (int k = 0; k < 4; k++) out[o++] = (uint8_t)(crc >> (8 * k));
    for (int k = 0; k < 4; k++) out[o++] = (uint8_t)((uint64_t)n >> (8 * k));
  }
  free(p.bout);
  free(p.blen);
  free(p.bcrc);
  pthread_mutex_destroy(&p.mu);
  return ok ? o : 0;
}

size_t syn_gzip_bound(size_t n) { return n + n / 1000 + (n / 16384 + 1) * 16 + 4096; }
