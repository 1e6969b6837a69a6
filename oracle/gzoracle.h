/*
 * gzoracle.h -- CPU oracle for the gzip decompression hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the byte-exact checker for the
 * CUDA path and the timed CPU baseline.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference arm may load it.  The product path
 * (gzippy_b200/, libgzgpu.so) never links or calls it.
 *
 * It restates the reference's (JackDanger/gzippy v0.8.0) decode algorithm in
 * plain C, function by function; each definition in gzoracle.c cites the
 * reference file:line it follows.  Parity is pinned by tests against the
 * reference's own GZBLK01 known-answer blocks (corpus/silesia_blocks) and
 * against system zlib 1.3 inflate.
 */
#ifndef GZORACLE_H
#define GZORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes shared with the C-ABI (include/gzgpu.h) */
enum {
  ORC_OK = 0,
  ORC_NOT_GZIP = 1,
  ORC_BAD_HEADER = 2,
  ORC_BAD_DEFLATE = 3,
  ORC_CRC_MISMATCH = 4,
  ORC_SIZE_MISMATCH = 5,
  ORC_OUT_TOO_SMALL = 6,
  ORC_TRUNCATED = 9,
};

/* flags of orc_inflate_chunk_ex */
enum {
  ORC_START_SYNC = 1,  /* a sync start: inside the block whose header is at start_table
                          (0: a non-final fixed-Huffman block) */
  ORC_ZERO_WINDOW = 2, /* back-references before the chunk read zeros (member start) */
};
#define ORC_SYNC_OFFSETS 64
#define ORC_SYNC_SPAN 8192
#define ORC_SYNC_SPAN_DYN 16384

/* window modes for orc_inflate_chunk */
enum {
  ORC_WIN_MARKERS = 0, /* window unknown: back-refs before the chunk emit u16 markers */
  ORC_WIN_BYTES = 1,   /* window known: `window` holds up to 32 KiB (zero padded on the left) */
};

typedef struct {
  uint64_t end_bit;       /* bit where decoding stopped (block boundary, or end of the final block) */
  uint64_t out_len;       /* entries written */
  uint64_t marker_end;    /* 1 + position of the last marker entry written (0 = none) */
  uint32_t n_blocks;
  uint32_t n_stored, n_fixed, n_dynamic; /* block-type histogram */
  int32_t final_block;    /* 1 if the BFINAL block was decoded */
  int32_t status;         /* ORC_OK / ORC_BAD_DEFLATE / ORC_TRUNCATED / ORC_OUT_TOO_SMALL */
} orc_chunk_result;

typedef struct {
  uint64_t start;         /* byte offset of the member's gzip header */
  uint64_t length;        /* bytes up to the next candidate (or end of data) */
  uint64_t deflate_start; /* byte offset of the raw deflate stream */
  uint32_t isize;         /* ISIZE read from the 4 bytes before the next candidate */
  uint32_t pad;
  uint64_t output_offset; /* prefix sum of isize */
} orc_member;

typedef struct {
  uint64_t n_chunks;         /* partitions in the grid */
  uint64_t n_candidates_ok;  /* partitions whose finder produced a start */
  uint64_t n_spec_rejected;  /* speculative chunks discarded by the chain check */
  uint64_t n_repairs;        /* confirmed re-decodes */
  uint64_t n_tail_marker_chunks;
  uint64_t n_members;
} orc_chunked_stats;

uint32_t orc_crc32(uint32_t crc, const uint8_t *p, size_t n);
uint32_t orc_crc32_combine(uint32_t crc1, uint32_t crc2, uint64_t len2);
uint32_t orc_gf2_mulmod(uint32_t a, uint32_t b);
uint32_t orc_x_pow_8n(uint64_t nbytes);

/* gzip header: returns ORC_OK and *hdr_len, or ORC_BAD_HEADER / ORC_TRUNCATED */
int orc_gzip_header(const uint8_t *p, size_t n, size_t *hdr_len);

/* block finder: every candidate with bit_offset in [start_bit, end_bit),
 * sorted by (bit_offset, seek_bit).  Returns the number written (<= cap). */
size_t orc_find_blocks(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t end_bit,
                       uint64_t *first, uint64_t *seek, size_t cap);
/* orc_find_blocks with the device's partition-start rule for stored
 * candidates: the block after one must be stored or a valid dynamic block. */
size_t orc_find_starts(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t end_bit,
                       uint64_t *first, uint64_t *seek, size_t cap);
/* dynamic-header predicate at one bit offset (1 = candidate) */
int orc_is_dynamic_candidate(const uint8_t *data, size_t n, uint64_t bit);

/* decode one chunk: from start_bit, stop at the first block boundary >= stop_lo,
 * or after the BFINAL block.  Output entries are u16 (markers >= 32768). */
int orc_inflate_chunk(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t stop_lo,
                      int window_mode, const uint8_t *window, size_t wlen, uint16_t *out,
                      size_t cap, orc_chunk_result *res);

/* code lengths of the dynamic block header at `bit` (litlen then dist) */
/* orc_inflate_chunk with sync-start modes (no reference counterpart; the
 * device decoder's sync starts): see gzoracle.c inflate_core.  *sync_end =
 * 1 when the chunk stopped at a sync target; *end_hdr = the header bit of
 * the block it stopped in (0 for a fixed sync start). */
int orc_inflate_chunk_ex(const uint8_t *data, size_t n, uint64_t start_bit, uint64_t stop_lo,
                         int flags, uint64_t start_table, const uint64_t *sync_targets,
                         const uint64_t *target_tables, size_t n_targets, uint16_t *out,
                         size_t cap, orc_chunk_result *res, uint32_t *sync_end,
                         uint64_t *end_hdr);
/* Sync start inside the dynamic block whose header is at table_bit. */
int orc_dyn_sync_find(const uint8_t *data, size_t n, uint64_t table_bit, uint64_t from,
                      uint64_t to, uint64_t *bit);
/* Sync start in fixed-Huffman data for the range [from, to): 1 and *bit, or 0. */
int orc_fixed_sync_find(const uint8_t *data, size_t n, uint64_t from, uint64_t to, uint64_t *bit);
int orc_dynamic_lengths(const uint8_t *data, size_t n, uint64_t bit, uint8_t *lens, int *nlen,
                        int *ndist);

/* member scan (restates scan_member_boundaries_fast) */
size_t orc_scan_members(const uint8_t *data, size_t n, orc_member *out, size_t cap);

/* whole-stream serial decode with reference semantics (members, CRC/ISIZE) */
int orc_decompress(const uint8_t *in, size_t n, uint8_t *out, size_t cap, size_t *out_len);

/* chunked speculative decode (finder + markers + window chain + resolve +
 * CRC combine) on `threads` host threads. */
int orc_decompress_chunked(const uint8_t *in, size_t n, size_t chunk_bytes, int threads,
                           uint8_t *out, size_t cap, size_t *out_len, orc_chunked_stats *st);

/* resolve u16 entries against a 32 KiB window (window[0] = oldest byte) */
void orc_resolve_markers(const uint16_t *in, size_t n, const uint8_t *window32k, uint8_t *out);

#ifdef __cplusplus
}
#endif
#endif
