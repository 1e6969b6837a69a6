/*
 * gzgpu.h -- C ABI of the B200 gzip decompression backend.
 *
 * Drop-in for the decompression path of gzippy (JackDanger/gzippy v0.8.0).
 * Each entry point names the reference interface it replaces (paths are
 * relative to the reference project root).  Plain pointers and sizes only.
 *
 * Stream semantics follow the reference: input that does not start with
 * the gzip magic 1f 8b yields GZGPU_NOT_GZIP and no output (the reference's
 * Ok(empty), src/lib.rs:50-52); members are decoded in order and every
 * member's CRC32 and ISIZE are verified; bytes after a member that do not
 * start another gzip header end the stream cleanly; corrupt or truncated
 * members are errors (src/decompress/mod.rs:742-870, tests/lib_api.rs:361-390).
 *
 * Threading: a context serialises its own calls (internal mutex); use one
 * context per host thread for concurrency.  All host buffers belong to the
 * caller; device buffers belong to the context.
 */
#ifndef GZGPU_H
#define GZGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The Rust shim maps GZGPU_NOT_GZIP to Ok(empty) and every
 * other non-zero code to GzippyError::Decompression(gzgpu_strerror(code))
 * (src/error.rs:7-46). */
#define GZGPU_OK 0
#define GZGPU_NOT_GZIP 1
#define GZGPU_BAD_HEADER 2
#define GZGPU_BAD_DEFLATE 3
#define GZGPU_CRC_MISMATCH 4
#define GZGPU_SIZE_MISMATCH 5
#define GZGPU_OUT_TOO_SMALL 6 /* *out_len holds the size needed */
#define GZGPU_DEVICE_ERROR 7
#define GZGPU_TIMEOUT 8
#define GZGPU_TRUNCATED 9
#define GZGPU_INVALID_ARGUMENT 12
#define GZGPU_NOALLOC_TOO_LARGE 14 /* output beyond GZGPU_NOALLOC_MAX_OUT */
#define GZGPU_OVER_BUDGET 15 /* request larger than the server's device-memory budget */
#define GZGPU_PENDING 16     /* gzgpu_poll: the request has not finished */

/* readable bytes the device-resident entry point needs after the input */
#define GZGPU_INPUT_PAD 1024

typedef struct gzgpu_ctx gzgpu_ctx;

typedef struct {
  int device;         /* CUDA device ordinal */
  size_t chunk_bytes; /* compressed bytes per speculative chunk; 0 = tuned default */
  int lut_bits;       /* litlen LUT index bits: 10, 11 or 12; 0 = tuned default */
  int autotune;       /* 1 = choose chunk_bytes, lut_bits and ctas_per_sm per job: the
                         first job of each kind (compressed-size bucket, stream-count
                         bucket, share of streams whose first block is fixed-Huffman)
                         is decoded once per candidate and the fastest is kept for
                         later jobs of that kind; overrides the three fields */
  int ring_history;   /* 1 = decode history in a shared-memory ring (3 warps/SM) instead
                         of the output pages in HBM (24 or 32 warps/SM, the default) */
  int ctas_per_sm;    /* page-history decoder: 3 (24 warps/SM, 80 registers; default) or
                         4 (32 warps/SM, 64 registers); 0 = default */
  int fine_split;     /* 1 = cut partitions whose first blocks promise a high output
                         ratio into pieces and give pieces without a block start a
                         sync start inside their dynamic block; 0 = off (default:
                         measured no faster on the mixed, multi-member and batch
                         workloads) */
  int high_priority;  /* 1 = the context's stream has the device's greatest priority:
                         its pending thread blocks are scheduled before those of other
                         contexts' streams (running blocks are not preempted) */
  int work_order;     /* order in which the persistent decoder takes chunks: 0 = longest
                         expected decode first (default), 1 = in stream order */
  int decoder;        /* Huffman block bodies: 0 = default (4), 1 = lane-parallel 32-bit steps
                         (each lane decodes a whole candidate symbol at one bit offset),
                         2 = warp-uniform serial decode, 3 = lane-parallel 64-bit steps (each
                         lane looks up literal codes at two bit offsets; length, end and
                         long codes are decoded on the chain walk by the whole warp),
                         4 = chosen per block: 3 where length codes take under 0.3 of the
                         code space (literal-heavy data), else 1 */
} gzgpu_config;

typedef struct {
  const uint8_t *data;
  size_t len;
} gzgpu_span;

typedef struct {
  uint8_t *data; /* caller buffer */
  size_t cap;
  size_t len;    /* set by the call: bytes written, or bytes needed (OUT_TOO_SMALL) */
} gzgpu_out;

typedef struct {
  double ms_total;      /* device time of the last call (CUDA events) */
  double ms_h2d, ms_scan, ms_find, ms_decode, ms_walk, ms_resolve, ms_crc, ms_d2h;
  double ms_decode_kernel; /* the persistent inflate kernel alone (all passes) */
  uint64_t in_bytes, out_bytes;
  uint64_t n_streams, n_members, n_chunks, n_accepted, n_rejected, n_repairs;
  uint64_t n_tail_marker_chunks, n_pages, decode_passes, kernel_launches;
  uint64_t chunk_bytes;
  int32_t lut_bits;
  int32_t ctas_per_sm;
  uint32_t tune_key;    /* autotuner key of the last job (0 when autotune is off) */
  uint32_t tune_trials; /* decodes the autotuner ran for the last call (0 = cached) */
  uint32_t pool_regrows; /* times the page pool was grown and the chunks that had run
                            out of pages were decoded again */
  uint32_t reserved;
} gzgpu_stats;

/* Create / destroy a context on cfg->device (NULL cfg = defaults). */
int gzgpu_create(gzgpu_ctx **out, const gzgpu_config *cfg);
void gzgpu_destroy(gzgpu_ctx *ctx);
const char *gzgpu_strerror(int code);

/* gzippy::decompress / decompress_with_threads (src/lib.rs:176,189):
 * host in -> host out.  The thread count of the reference has no meaning on
 * the device and is not taken.  On GZGPU_OUT_TOO_SMALL *out_len is the
 * size needed. */
int gzgpu_decompress(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len, uint8_t *out,
                     size_t out_cap, size_t *out_len);

/* gzippy::decompress_raw / deflate_decode (src/lib.rs:250; decompress_raw_bytes,
 * src/decompress/mod.rs:920): one raw DEFLATE stream (RFC 1951, no gzip
 * header or trailer), decoded up to its final block; bytes after it are
 * ignored.  No checksum exists to verify.  Empty or cut-off input:
 * GZGPU_TRUNCATED; invalid DEFLATE: GZGPU_BAD_DEFLATE.  On
 * GZGPU_OUT_TOO_SMALL *out_len is the size needed. */
int gzgpu_inflate_raw(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len, uint8_t *out,
                      size_t out_cap, size_t *out_len);

/* decompress_zlib_turbo (src/decompress/mod.rs:895-914): zlib data decoded
 * as the raw DEFLATE stream between its 2-byte header and 4-byte Adler-32
 * trailer; like the reference, neither is checked.  Fewer than 6 bytes:
 * GZGPU_INVALID_ARGUMENT; otherwise as gzgpu_inflate_raw. */
int gzgpu_inflate_zlib(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len, uint8_t *out,
                       size_t out_cap, size_t *out_len);

/* gzippy's seek index (build_index + serialize_index, src/decompress/index.rs:
 * 55-141; checkpoint rule of scan_deflate, src/decompress/scan_inflate.rs:
 * 46-130), built from the parallel decode: at each DEFLATE block start whose
 * output offset has reached the next checkpoint (interval_bytes after the
 * previous one) and at least 32 KiB, a point records the header's bit offset
 * from the deflate start, the output offset and the 32 KiB of output before
 * it.  Written in the index format's version 1 layout ("GZIDX\x01", the
 * layout load_index reads with a bit offset per point).  Single-member gzip
 * only: other input gives GZGPU_INVALID_ARGUMENT, as in the reference.  On
 * GZGPU_OUT_TOO_SMALL *index_len is the size needed. */
int gzgpu_build_index(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len, uint64_t interval_bytes,
                      uint8_t *index_out, size_t index_cap, size_t *index_len);

/* gzippy::decompress_to_writer / _with_threads (src/lib.rs:204,221):
 * output delivered in order through `write` (return 0 to continue, non-zero
 * to abort with GZGPU_INVALID_ARGUMENT); *written = total bytes delivered. */
typedef int (*gzgpu_write_fn)(void *user, const uint8_t *data, size_t len);
int gzgpu_decompress_to_writer(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len,
                               gzgpu_write_fn write, void *user, uint64_t *written);

/* Device-resident form of gzgpu_decompress (internal decompress_bytes,
 * src/decompress/mod.rs:317): d_in / d_out are device pointers of this
 * context's device, both 16-byte aligned (cudaMalloc memory is); d_in must
 * have GZGPU_INPUT_PAD readable bytes past in_len.  No host copies of
 * payload. */
int gzgpu_decompress_device(gzgpu_ctx *ctx, const void *d_in, size_t in_len, void *d_out,
                            size_t out_cap, size_t *out_len);

/* Many independent streams in one job (no reference counterpart: the
 * reference decodes one stream per call).  statuses[i] / outs[i].len per
 * stream; returns GZGPU_OK when every stream decoded (or was not gzip). */
int gzgpu_decompress_batch(gzgpu_ctx *ctx, const gzgpu_span *ins, size_t n, gzgpu_out *outs,
                           int *statuses);

/* Device-resident form of gzgpu_decompress_batch (no reference
 * counterpart): n streams already in device memory at d_in + in_offs[i]
 * (offsets multiples of 16, host arrays), GZGPU_INPUT_PAD readable bytes
 * past the end of the last stream.  All streams decode in one job and land
 * back to back in d_out in stream order: out_offs[i] / out_lens[i] (host
 * arrays) give each stream's range, statuses[i] its status.  Returns
 * GZGPU_OK, the first failing stream's status, or GZGPU_OUT_TOO_SMALL when
 * the total exceeds out_cap (then out_lens hold the sizes needed). */
int gzgpu_decompress_batch_device(gzgpu_ctx *ctx, const void *d_in, const uint64_t *in_offs,
                                  const uint64_t *in_lens, size_t n, void *d_out, size_t out_cap,
                                  uint64_t *out_offs, uint64_t *out_lens, int *statuses);

/* Decode without allocating (no counterpart in the reference).
 *
 * For callers that cannot call cudaMalloc: code under a pool-only allocator
 * that must not grow, real-time paths that cannot absorb the device-wide
 * synchronisation cudaMalloc/cudaFree may cause, and processes whose device
 * memory is all reserved up front by another framework.  Needs no context:
 * it runs on the current device and the caller's stream (`cuda_stream`,
 * a cudaStream_t; NULL = the default stream), with d_in / d_out in device
 * memory (d_in 4-byte aligned with GZGPU_INPUT_PAD readable bytes past
 * in_len).  It calls no cudaMalloc, cudaFree or allocating library routine.
 *
 * Its working memory is one file-scope device array of about 8.5 MiB that
 * every GPU loading this library holds until the process exits; so the
 * output of one call is limited to GZGPU_NOALLOC_MAX_OUT bytes (4 MiB, all
 * members together) and larger streams return GZGPU_NOALLOC_TOO_LARGE.  One
 * warp decodes the members in order (no speculative chunks): made for small
 * streams, not throughput.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls share the array: calls whose work overlaps on the GPU
 * (on different streams, or from different threads) race and must not be
 * issued; calls ordered on one stream are fine.  The call waits for its
 * stream to finish the decode and returns the status; *out_len = bytes
 * written, or on GZGPU_OUT_TOO_SMALL the exact size of the whole stream
 * (every member is still decoded and checked; members from the first one
 * that does not fit are not written).  The launch's own failure returns
 * GZGPU_DEVICE_ERROR; the thread's last-error state is left as it was. */
#define GZGPU_NOALLOC_MAX_OUT (4u << 20)
int gzgpu_decompress_device_noalloc(const void *d_in, size_t in_len, void *d_out, size_t out_cap,
                                    size_t *out_len, void *cuda_stream);

/* Serving (no reference counterpart): a continuous-batching service over
 * host buffers.  Requests are submitted from any thread and decoded by
 * `lanes` worker threads, each with its own context (CUDA stream and device
 * buffers kept between batches), so batches overlap on the GPU.  A request
 * is admitted when its charge (compressed size + 3 x out_cap + 1 MiB: output
 * and decoder pages) fits the device-memory budget next to the requests in
 * flight; the queue is FIFO.  A request of at least large_bytes compressed
 * runs alone; smaller ones are merged, up to max_batch_bytes of input, into
 * one batch (one gzgpu_decompress_batch job).  small_lanes of the lanes take
 * only small requests, so these never wait behind large ones.  Inputs and outputs are the
 * caller's and must stay valid until the request has been polled done. */
typedef struct gzgpu_server gzgpu_server;

typedef struct {
  int device;
  int lanes;                 /* concurrent batches; 0 = 4 */
  int autotune;              /* the lanes' contexts use the autotuner */
  int small_lanes;           /* lanes that take only small requests; 0 = 1 (with 2+ lanes),
                                -1 = none */
  size_t budget_bytes;       /* device-memory budget of admitted requests; 0 = 120 GB */
  size_t max_batch_bytes;    /* compressed bytes merged into one batch; 0 = 256 MiB */
  size_t max_batch_requests; /* requests merged into one batch; 0 = 4096 */
  size_t large_bytes;        /* compressed size from which a request runs alone; 0 = 32 MiB */
} gzgpu_server_config;

typedef struct {
  double queue_ms;  /* submit -> admitted to a lane */
  double total_ms;  /* submit -> decoded (host output written) */
} gzgpu_request_times;

typedef struct {
  uint64_t submitted, completed, batches, in_flight, queued, budget_used, in_bytes, out_bytes;
} gzgpu_server_stats;

int gzgpu_server_create(gzgpu_server **out, const gzgpu_server_config *cfg);
/* Waits for running batches; requests still queued are dropped. */
void gzgpu_server_destroy(gzgpu_server *srv);
/* Queue one gzip buffer; *ticket identifies it.  GZGPU_OVER_BUDGET when its
 * charge alone exceeds the budget. */
int gzgpu_submit(gzgpu_server *srv, const uint8_t *in, size_t in_len, uint8_t *out,
                 size_t out_cap, uint64_t *ticket);
/* GZGPU_PENDING while the request runs (wait_ms: 0 = return at once, < 0 =
 * wait until done, > 0 = wait at most that long); then its status (as
 * gzgpu_decompress), *out_len and its times, and the ticket is released. */
int gzgpu_poll(gzgpu_server *srv, uint64_t ticket, int wait_ms, size_t *out_len,
               gzgpu_request_times *times);
int gzgpu_server_get_stats(gzgpu_server *srv, gzgpu_server_stats *out);

/* Diagnostics (no reference counterpart; used by the parity tests).
 *
 * gzgpu_debug_find: run the block-finder kernel on `in` for n ranges
 * [from[i], to[i]) (bit offsets); lo/hi = first candidate's (bit_offset,
 * seek_bit), valid[i] = 0 when the range holds none, 1 for a block header,
 * 2 for a sync start in fixed-Huffman data (lo = hi = its bit; no
 * reference counterpart).  Mirrors DeflateBlockValidator::find_first_candidate
 * (src/decompress/parallel/blockfinder_validation.rs:319).
 *
 * gzgpu_debug_decode: run the inflate kernel on n explicit chunks (start
 * bit, stop bit, flags[i]: bit 0 = member start (zero window instead of
 * markers), bit 1 = sync start, inside the block whose header is at
 * table_bit[i] (NULL or 0 = a fixed block)) and copy each chunk's u16
 * entries to entries + i*cap_per.  A chunk followed by sync starts may stop
 * at them mid-block.  res[7*i..] = end_bit, out_len, marker_end, n_blocks, status,
 * final_block, sync_end.  Mirrors decode_chunk
 * (src/decompress/parallel/chunk_decode.rs:225). */
int gzgpu_debug_find(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len, const uint64_t *from,
                     const uint64_t *to, size_t n, uint64_t *lo, uint64_t *hi, int *valid);
int gzgpu_debug_decode(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len, const uint64_t *start,
                       const uint64_t *stop, const int *flags, size_t n, uint16_t *entries,
                       size_t cap_per, uint64_t *res, const uint64_t *table_bit);
/* gzgpu_debug_dyn_sync: the dynamic sync-start search for n ranges
 * [from[i], to[i]) inside the block whose header is at table_bit[i]; out[i]
 * = the start found, valid[i] = 1 when one was found. */
int gzgpu_debug_dyn_sync(gzgpu_ctx *ctx, const uint8_t *in, size_t in_len, const uint64_t *table_bit,
                         const uint64_t *from, const uint64_t *to, size_t n, uint64_t *out,
                         int *valid);

/* gzgpu_debug_last_chunks: the chunk table of the last job.  descs holds
 * n records of 80 bytes (start_bit, lo_bit, stop_lo, guess_bit, limit_bit,
 * in_end, abort_bit, table_bit as u64; flags, stream, next as u32,
 * est_ratio as f32); results n records of 80 bytes (end_bit, out_len,
 * marker_end as u64; last_page, prev_page, n_pages, n_blocks as u32;
 * status, final_block as i32; t_start, t_end as u64 device nanoseconds;
 * gen, sync_end as u32; end_hdr_bit as u64).  *n = records available
 * (copies min(cap, *n)). */
int gzgpu_debug_last_chunks(gzgpu_ctx *ctx, void *descs, void *results, size_t cap, size_t *n);

/* Statistics of the last call. */
int gzgpu_get_stats(gzgpu_ctx *ctx, gzgpu_stats *out);

#ifdef __cplusplus
}
#endif
#endif /* GZGPU_H */
