// common.cuh -- device/host shared definitions for the gzip decode kernels.
//
// Data layout in HBM (one decode job = one stream, a batch of streams, or a
// serving tick):
//   input    : every stream's gzip bytes back to back, + kInputPad zero bytes
//   chunks   : ChunkDesc[] (what to decode) and ChunkResult[] (what came out)
//   pages    : PagePool, fixed pages of kPageEntries u16 entries; a chunk's
//              decoded entries (bytes < 256, window markers >= 32768) live in
//              the pages it allocated, in allocation order
//   output   : final bytes, one contiguous range per stream
#pragma once
#include <cstdint>

namespace gzgpu {

constexpr uint32_t kWindow = 32768;          // deflate window (entries)
constexpr uint32_t kRingMask = kWindow - 1;  // decoder history ring = one window
constexpr uint32_t kMarkerBase = 32768;      // entry >= kMarkerBase: window index + 32768
constexpr uint32_t kPageEntries = 65536;     // u16 entries per output page
constexpr uint32_t kFlush = 8192;            // ring -> page flush unit (entries)
constexpr uint32_t kInputPad = 1024;         // zero bytes after the input buffer
constexpr uint64_t kNoStop = ~0ull;
constexpr uint64_t kNoTrailer = ~0ull;  // a member without CRC32/ISIZE (raw DEFLATE)
constexpr uint32_t kNoPage = 0xFFFFFFFFu;

// status codes (same numbering as include/gzgpu.h)
enum : int32_t {
  kOk = 0,
  kNotGzip = 1,
  kBadHeader = 2,
  kBadDeflate = 3,
  kCrcMismatch = 4,
  kSizeMismatch = 5,
  kOutTooSmall = 6,
  kDeviceError = 7,
  kTimeout = 8,
  kTruncated = 9,
  kPoolExhausted = 10,
  kNotDecoded = 11,
  kOvershoot = 13,  // speculative chunk ran past stop_lo + slack without a block boundary
  kNoAllocTooLarge = 14,  // output beyond the no-allocation entry point's limit
};

enum : uint32_t {
  kChunkMemberFirst = 1u,  // starts a member: zero window, never emits markers
  kChunkValid = 2u,        // has a start (member start or a finder candidate)
  kChunkConfirmed = 4u,    // starts at a boundary the chain walk confirmed (a repair)
  kChunkSync = 8u,         // a sync start: a symbol boundary inside a Huffman block, not
                           // a block header (table_bit: that block's header; 0 = a
                           // non-final fixed-Huffman block)
  kChunkPiece = 16u,       // a piece of a partition cut by its output estimate
};
// flags bits 24..31: the chunk's first decode attempt number (its pages carry
// attempt numbers from there; raised when a chunk is decoded again after the
// page pool ran out, so its old pages never pass for the new ones)
constexpr int kGenBaseShift = 24;
constexpr uint32_t kGenBaseMax = 255;

// Sync starts in fixed-Huffman data: positions are walked from kSyncOffsets
// consecutive start bits to the first symbol boundary at or past
// from + kSyncOffsets + kSyncSpan.
constexpr uint32_t kSyncOffsets = 64;
constexpr uint64_t kSyncSpan = 8192;
constexpr uint64_t kSyncSpanDyn = 16384;  // walk length inside a dynamic block
constexpr uint64_t kSyncMinSlack = 1ull << 16;  // least run past its stop of a sync start
constexpr uint64_t kSyncFail = ~0ull;

struct ChunkDesc {
  uint64_t start_bit;  // absolute bit offset in the input buffer to decode from
  uint64_t lo_bit;     // earliest acceptable start (stored-block padding), <= start_bit
  uint64_t stop_lo;    // stop at the first block boundary >= stop_lo
  uint64_t guess_bit;  // partition start the finder searched from
  uint64_t limit_bit;  // end of the finder's search range
  uint64_t in_end;     // byte end of this chunk's stream in the input buffer
  uint64_t abort_bit;  // a speculative chunk gives up past this bit (kNoStop = never)
  uint64_t table_bit;  // sync start: header bit of its block (0 = fixed code, or none)
  uint32_t flags;
  uint32_t stream;     // stream id
  uint32_t next;       // index of the next valid chunk of the stream (kNoChunk = none)
  float est_ratio;     // finder's estimate of output bytes per input byte (0 = none)
};
constexpr uint32_t kNoChunk = 0xFFFFFFFFu;
// phantom successors a speculative chunk decodes through; a chunk whose start
// is certain (member-first or confirmed) decodes through any number of them
constexpr int kMaxExtends = 4;

struct ChunkResult {
  uint64_t end_bit;     // bit where decoding stopped
  uint64_t out_len;     // entries produced
  uint64_t marker_end;  // 1 + last marker position (0 = no markers)
  uint32_t last_page;
  uint32_t prev_page;
  uint32_t n_pages;
  uint32_t n_blocks;
  int32_t status;
  int32_t final_block;
  uint64_t t_start, t_end;  // %globaltimer (ns) when the warp took / finished the chunk
  uint32_t gen;             // decode attempt that produced this result (page tag)
  uint32_t sync_end;        // 1: stopped at its successor's sync start (mid-block)
  uint64_t end_hdr_bit;     // sync_end: header bit of the block it stopped in (0 = fixed)
};

// a page's seq word: attempt (gen) in the top 8 bits, page index below
constexpr uint32_t kSeqMask = 0x00FFFFFFu;
constexpr int kGenShift = 24;
constexpr uint32_t kMaxTries = 4;  // speculative starts tried per chunk

// one DEFLATE block a chunk decoded (seek-index builds only): where its
// header starts and how much output the chunk had produced before it
struct BlockRec {
  uint64_t hdr_bit;  // absolute input bit of the block header
  uint64_t out_pos;  // chunk-local output position at the block's start
  uint32_t chunk, gen;
};

struct PagePool {
  uint16_t* data;    // cap * kPageEntries entries
  uint32_t* owner;   // chunk id per page
  uint32_t* seq;     // page index within its chunk
  uint32_t* next;    // allocation counter
  uint32_t cap;
  // block log: null unless a seek index is being built
  BlockRec* blocks = nullptr;
  uint32_t* n_blocks = nullptr;
  uint32_t blocks_cap = 0;
  // Huffman block bodies: 0 = lane-parallel 32-bit steps, 1 = warp-uniform
  // serial, 2 = lane-parallel 64-bit steps with matches decoded on the walk,
  // 3 = per block, 2 for literal-heavy blocks and 0 for the others
  uint32_t serial = 0;
};

// resolve plan entry: one accepted chunk in output order
struct PlacedChunk {
  uint64_t out_off;      // final output offset of entry 0
  uint64_t member_off;   // final output offset where the chunk's member begins
  uint32_t chunk;        // chunk id
  uint32_t pad;
};

// CRC block: a run of final output bytes inside one member
struct CrcBlock {
  uint64_t off;
  uint32_t len;
  uint32_t member;
};

}  // namespace gzgpu
