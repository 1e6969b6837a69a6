// resolve.cu -- window propagation, marker resolution and CRC32 (K3-K5).
//
// After decoding, every accepted chunk k has an output offset out_off[k]
// and u16 entries in its pages.  An entry v < 256 is a byte; v >= 32768 is
// window index v - 32768 of the 32 KiB that precede the chunk in the final
// output (replace_markers.rs:7-23), i.e. final[out_off - 32768 + v - 32768],
// read as 0 before the member's first byte (the zero window).
//
//   tail_literals : bytes of every chunk's last 32 KiB ("tail") -> output
//   tail_markers  : markers in tails, chunk after chunk in output order: a
//                   tail's markers only reach the tails of earlier chunks,
//                   so this walk is the window chain (window_map.rs:80-103,
//                   chunk_fetcher.rs publish_subchunk_windows :2295)
//   body          : all other entries, fully parallel over pages, reading
//                   windows the chain made final (resolve_and_narrow_markers
//                   _in_place_crc, chunk_data.rs:1745)
//   crc_blocks    : CRC32 of blocks of final output (up to 32 KiB of one
//                   member each), each block's CRC moved to its member's end
//                   and XORed into the member's register (crc32.rs
//                   combine_crc32 :127 combines the same quantities)
//   member_check  : each member's CRC32 and ISIZE against its trailer
#include <cstdint>

#include "common.cuh"
#include "resolve.cuh"

namespace gzgpu {

// page of entry q of a chunk's last 32 KiB: the page of its last entry or
// the one before (a page holds 64 Ki entries)
__device__ __forceinline__ const uint16_t* chunk_entry_page(const ChunkResult& r, uint64_t q,
                                                            const PagePool& pool) {
  uint64_t last_seq = (r.out_len - 1) / kPageEntries;
  uint32_t page = (q / kPageEntries == last_seq) ? r.last_page : r.prev_page;
  return pool.data + (size_t)page * kPageEntries;
}

// One warp writes the bytes of a span of 32 groups of 4 entries: lane L
// holds the bytes of entries 4L .. 4L + 3 of the span in `w` (byte j of w =
// entry 4L + j) and in `valid` which of them to write; `d0` is the output
// address of the span's entry 0.  Each lane stores the aligned 32-bit word
// that starts inside its group (its last bytes, then the next lane's first,
// by a funnel shift), so a warp writes 128 contiguous bytes per store; bytes
// of partly valid words and the two words the span shares with its
// neighbours go out one by one.
__device__ __forceinline__ void warp_store_bytes(uint8_t* __restrict__ out, uint64_t d0, uint32_t w,
                                                 uint32_t valid, int lane) {
  const uint32_t s = (uint32_t)(d0 & 3);
  const uint64_t dl = d0 + 4 * (uint64_t)lane;
  if (s == 0) {
    if (valid == 0xFu) {
      *reinterpret_cast<uint32_t*>(out + dl) = w;
    } else {
      for (int j = 0; j < 4; j++)
        if ((valid >> j) & 1) out[dl + j] = (uint8_t)(w >> (8 * j));
    }
    return;
  }
  const uint32_t u = 4 - s;  // bytes of this group before the next aligned word
  const uint32_t wn = __shfl_down_sync(0xFFFFFFFFu, w, 1);
  const uint32_t vn = __shfl_down_sync(0xFFFFFFFFu, valid, 1);
  if (lane < 31) {
    const uint32_t vw = (valid >> u) | ((vn << s) & 0xFu);
    const uint32_t ww = __funnelshift_r(w, wn, 8 * u);
    if (vw == 0xFu) {
      *reinterpret_cast<uint32_t*>(out + dl + u) = ww;
    } else {
      for (int j = 0; j < 4; j++)
        if ((vw >> j) & 1) out[dl + u + j] = (uint8_t)(ww >> (8 * j));
    }
  } else {
    for (uint32_t j = u; j < 4; j++)
      if ((valid >> j) & 1) out[dl + j] = (uint8_t)(w >> (8 * j));
  }
  if (lane == 0)
    for (uint32_t j = 0; j < u; j++)
      if ((valid >> j) & 1) out[dl + j] = (uint8_t)(w >> (8 * j));
}

// the 4 entries of a group (page-relative index e, a multiple of 4)
__device__ __forceinline__ void load_group(const uint16_t* page, uint32_t e, uint32_t v[4]) {
  const uint2 x = *reinterpret_cast<const uint2*>(page + e);
  v[0] = x.x & 0xFFFFu;
  v[1] = x.x >> 16;
  v[2] = x.y & 0xFFFFu;
  v[3] = x.y >> 16;
}

// one CTA per chunk: the bytes of its last 32 KiB (markers written as 0,
// which tail_markers_kernel replaces)
__global__ void tail_literals_kernel(const PlacedChunk* __restrict__ placed, uint32_t n,
                                     const ChunkResult* __restrict__ results, PagePool pool,
                                     uint8_t* __restrict__ out) {
  const uint32_t k = blockIdx.x;
  if (k >= n) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const PlacedChunk pc = placed[k];
  const ChunkResult r = results[pc.chunk];
  const uint64_t len = r.out_len, t0 = len > kWindow ? len - kWindow : 0;
  const uint64_t g0 = t0 & ~3ull;  // groups start at multiples of 4 (never across a page)
  for (uint64_t base = g0 + 128 * (uint64_t)warp; base < len; base += 128 * (uint64_t)nwarps) {
    const uint64_t q = base + 4 * (uint64_t)lane;
    uint32_t w = 0, valid = 0;
    if (q < len) {
      uint32_t v[4];
      load_group(chunk_entry_page(r, q, pool), (uint32_t)(q % kPageEntries), v);
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (q + j >= t0 && q + j < len) {
          valid |= 1u << j;
          w |= (v[j] < 256 ? v[j] : 0u) << (8 * j);
        }
    }
    warp_store_bytes(out, pc.out_off + base, w, valid, lane);
  }
}

// The markers of chunk tails.  A tail marker names a byte of the 32 KiB
// before its chunk, which lies in the tails of earlier chunks of the member
// (a chunk shorter than 32 KiB is all tail); that entry is a literal or
// again a marker, naming a byte before its own chunk.  Each marker follows
// its references through the chunks' entries until it reaches a literal (or
// a position before the member: 0), so all tails resolve in parallel: one
// CTA per chunk of the list (the chunks whose tails hold markers), placed
// chunks in output order.
__global__ void tail_markers_kernel(const PlacedChunk* __restrict__ placed,
                                    const uint32_t* __restrict__ list, uint32_t n_list,
                                    const ChunkResult* __restrict__ results, PagePool pool,
                                    uint8_t* __restrict__ out) {
  for (uint32_t i = blockIdx.x; i < n_list; i += gridDim.x) {
    const uint32_t k = list[i];
    const PlacedChunk pc = placed[k];
    const ChunkResult r = results[pc.chunk];
    const uint64_t len = r.out_len, t0 = len > kWindow ? len - kWindow : 0;
    const uint64_t end = r.marker_end < len ? r.marker_end : len;
    const int64_t moff = (int64_t)pc.member_off;
    for (uint64_t q = t0 + threadIdx.x; q < end; q += blockDim.x) {
      uint32_t v = chunk_entry_page(r, q, pool)[q % kPageEntries];
      if (v < kMarkerBase) continue;  // a literal: written by tail_literals_kernel
      uint32_t j = k;
      int64_t off = (int64_t)pc.out_off;
      uint32_t b = 0;
      for (;;) {
        const int64_t src = off - (int64_t)kWindow + (int64_t)(v - kMarkerBase);
        if (src < moff) break;  // before the member: the zero window
        // the chunk that holds src: one of the few before chunk j
        do {
          j--;
        } while ((int64_t)placed[j].out_off > src);
        const PlacedChunk pj = placed[j];
        const ChunkResult rj = results[pj.chunk];
        const uint64_t qj = (uint64_t)(src - (int64_t)pj.out_off);
        v = chunk_entry_page(rj, qj, pool)[qj % kPageEntries];
        if (v < kMarkerBase) {
          b = v;
          break;
        }
        off = (int64_t)pj.out_off;  // a marker of chunk j: its window is before chunk j
      }
      out[pc.out_off + q] = (uint8_t)b;
    }
  }
}

// one CTA per page: the entries before the chunk's tail, markers gathered
// from the final window; 4 entries per lane, aligned 32-bit stores
__global__ void body_kernel(const PlacedChunk* __restrict__ placed,
                            const uint32_t* __restrict__ placed_of_chunk, uint32_t n_pages,
                            const ChunkResult* __restrict__ results, PagePool pool,
                            uint8_t* __restrict__ out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (uint32_t p = blockIdx.x; p < n_pages; p += gridDim.x) {
    const uint32_t cid = pool.owner[p];
    const uint32_t k = placed_of_chunk[cid];
    if (k == 0xFFFFFFFFu) continue;
    const uint32_t sw = pool.seq[p];
    if ((sw >> kGenShift) != results[cid].gen) continue;  // page of a failed attempt
    const PlacedChunk pc = placed[k];
    const uint64_t len = results[cid].out_len;
    const uint64_t t0 = len > kWindow ? len - kWindow : 0;
    const uint64_t q0 = (uint64_t)(sw & kSeqMask) * kPageEntries;
    if (q0 >= t0) continue;
    const uint32_t n = (uint32_t)min((uint64_t)kPageEntries, t0 - q0);
    const uint16_t* src = pool.data + (size_t)p * kPageEntries;
    const int64_t wbase = (int64_t)pc.out_off - (int64_t)kWindow - (int64_t)kMarkerBase;
    const int64_t moff = (int64_t)pc.member_off;
    for (uint32_t base = 128 * warp; base < n; base += 128 * nwarps) {
      const uint32_t e = base + 4 * lane;
      uint32_t w = 0, valid = 0;
      if (e < n) {
        uint32_t v[4];
        load_group(src, e, v);
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (e + j < n) {
            valid |= 1u << j;
            uint32_t b = v[j];
            if (b >= 256) {
              const int64_t sidx = wbase + b;
              b = sidx >= moff ? out[sidx] : 0u;
            }
            w |= b << (8 * j);
          }
      }
      warp_store_bytes(out, pc.out_off + q0 + base, w, valid, lane);
    }
  }
}

// ---------------------------------------------------------------------------
// CRC32 (reflected 0xEDB88320).  A CRC register s followed by n zero bytes
// becomes A^n(s) = s * x^(8n) mod P (linear in s), so
//   raw(M1 | M2) = A^|M2|(raw(M1)) ^ raw(M2)       (raw: register starts at 0)
//   crc(M)       = ~(A^|M|(0xFFFFFFFF) ^ raw(M))
// and leading zero bytes leave raw() unchanged (crc32.rs combine_crc32 :127
// combines the same quantities).  Each block's raw CRC is moved to its
// member's end with A^(bytes after the block) and XORed into the member's
// register, so blocks fold in independently, in any order.
// ---------------------------------------------------------------------------
__device__ uint32_t d_crc_tab[4][256];  // slice-by-4 tables
__device__ uint32_t d_x2n[64];          // x^(2^k) mod P
// d_crc_shift[j][k][v] = A^(kCrcSlice << j)(v << 8k): moves a register past
// 2^j lane slices of zero bytes with 4 lookups
__device__ uint32_t d_crc_shift[kCrcLevels][4][256];

__device__ __forceinline__ uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
  uint32_t r = 0;
#pragma unroll 8
  for (int i = 31; i >= 0; i--) {
    r ^= b & (0u - ((a >> i) & 1u));
    b = (b >> 1) ^ (0xEDB88320u & (0u - (b & 1u)));
  }
  return r;
}

// x^(8n) mod P
__device__ __forceinline__ uint32_t x_pow_8n(uint64_t n) {
  uint32_t p = 1u << 31;
  uint64_t e = n << 3;
  for (int k = 0; e; e >>= 1, k++)
    if (e & 1) p = gf2_mulmod(d_x2n[k & 63], p);
  return p;
}

// x^(8n) mod P computed by a whole warp: lane k takes exponent bits k and
// k + 32, then a product tree over the lanes (every lane gets the result)
__device__ __forceinline__ uint32_t x_pow_8n_warp(uint64_t n, int lane) {
  const uint64_t e = n << 3;
  uint32_t f = 1u << 31;
  if ((e >> lane) & 1) f = d_x2n[lane];
  if ((e >> (lane + 32)) & 1) f = gf2_mulmod(f, d_x2n[lane + 32]);
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) f = gf2_mulmod(f, __shfl_xor_sync(0xFFFFFFFFu, f, d));
  return f;
}

__global__ void crc_init_kernel() {
  uint32_t i = threadIdx.x;
  uint32_t c = i;
  for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
  d_crc_tab[0][i] = c;
  __syncthreads();
  for (int t = 1; t < 4; t++) {
    uint32_t p = d_crc_tab[t - 1][i];
    d_crc_tab[t][i] = (p >> 8) ^ d_crc_tab[0][p & 0xFF];
    __syncthreads();
  }
  if (i == 0) {
    uint32_t v = 1u << 30;  // x^1
    for (int k = 0; k < 64; k++) {
      d_x2n[k] = v;
      v = gf2_mulmod(v, v);
    }
  }
}

// one block per (level, byte slot): 256 register values each
__global__ void crc_shift_init_kernel() {
  const uint32_t j = blockIdx.x >> 2, k = blockIdx.x & 3, v = threadIdx.x;
  const uint32_t xp = x_pow_8n((uint64_t)kCrcSlice << j);
  d_crc_shift[j][k][v] = gf2_mulmod(xp, v << (8 * k));
}

// the register s moved past 2^j lane slices, from the shift tables in shared memory
__device__ __forceinline__ uint32_t crc_shift(const uint32_t* shf, uint32_t s, int j) {
  const uint32_t* t = shf + j * 1024;
  return t[s & 0xFF] ^ t[256 + ((s >> 8) & 0xFF)] ^ t[512 + ((s >> 16) & 0xFF)] ^ t[768 + (s >> 24)];
}

// one byte into a CRC register, from the lane's own copy of the byte table
// (word 32 * index + lane of the shared array: every lane of a warp reads
// its own bank)
__device__ __forceinline__ uint32_t crc_byte(const uint32_t* ltab, uint32_t lane, uint32_t c,
                                             uint32_t b) {
  return ltab[(((c ^ b) & 0xFFu) << 5) | lane] ^ (c >> 8);
}

// CRC32 of the final output, one warp per block of up to kCrcBlock bytes of
// one member.  The block is cut into 32 lane slices of kCrcSlice bytes
// counted back from its end, so every slice has the same length once the
// bytes before the block count as zeros (they leave the register at 0).
// Each lane folds its slice byte by byte with its own copy of the byte
// table (no bank conflicts), reading aligned 16-byte words; the slices'
// registers merge in a tree of fixed shifts, and the block's register,
// moved past the rest of its member, is XORed into mem_raw.
__global__ void __launch_bounds__(kCrcThreads)
    crc_blocks_kernel(const CrcBlock* __restrict__ blocks, uint32_t n,
                      const uint8_t* __restrict__ out, const uint64_t* __restrict__ mem_end,
                      uint32_t* __restrict__ mem_raw) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint32_t* ltab = sm;              // [256][32] lane copies of the byte table
  uint32_t* shf = sm + 256 * 32;    // [kCrcLevels][4][256] shift tables
  for (uint32_t i = threadIdx.x; i < 256 * 32; i += kCrcThreads) ltab[i] = d_crc_tab[0][i >> 5];
  for (uint32_t i = threadIdx.x; i < kCrcLevels * 4 * 256; i += kCrcThreads)
    shf[i] = d_crc_shift[i >> 10][(i >> 8) & 3][i & 255];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (uint32_t bi = (blockIdx.x * kCrcThreads + threadIdx.x) >> 5; bi < n;
       bi += (gridDim.x * kCrcThreads) >> 5) {
    const CrcBlock blk = blocks[bi];
    const uint8_t* p = out + blk.off;
    const uint8_t* end = p + blk.len;
    // lane slice [s0, s1), clipped to the block
    const int64_t back = (int64_t)kCrcSlice * (32 - lane);
    const uint8_t* s1 = end - (back - kCrcSlice);
    const uint8_t* s0 = (int64_t)blk.len > back - kCrcSlice ? (back <= (int64_t)blk.len ? end - back : p) : s1;
    uint32_t c = 0;
    const uint8_t* q = s0;
    // bytes up to the first 16-byte boundary
    while (q < s1 && (reinterpret_cast<uintptr_t>(q) & 15)) c = crc_byte(ltab, lane, c, *q++);
    // aligned 16-byte words, the next one loaded while this one folds
    if (q + 16 <= s1) {
      uint4 w = *reinterpret_cast<const uint4*>(q);
      for (;;) {
        const bool more = q + 32 <= s1;
        uint4 nx = more ? *reinterpret_cast<const uint4*>(q + 16) : make_uint4(0, 0, 0, 0);
        const uint32_t wd[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
          c = crc_byte(ltab, lane, c, wd[k]);
          c = crc_byte(ltab, lane, c, wd[k] >> 8);
          c = crc_byte(ltab, lane, c, wd[k] >> 16);
          c = crc_byte(ltab, lane, c, wd[k] >> 24);
        }
        q += 16;
        if (!more) break;
        w = nx;
      }
    }
    while (q < s1) c = crc_byte(ltab, lane, c, *q++);
    // slices merge: 2^j slices on each side at level j
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const uint32_t r = __shfl_down_sync(0xFFFFFFFFu, c, 1 << j);
      if ((lane & ((2 << j) - 1)) == 0) c = crc_shift(shf, c, j) ^ r;
    }
    // move the block's register past the rest of its member
    const uint32_t xp = x_pow_8n_warp(mem_end[blk.member] - (blk.off + blk.len), lane);
    if (lane == 0) atomicXor(mem_raw + blk.member, gf2_mulmod(xp, c));
  }
}

// one thread per member: its CRC from the accumulated blocks, checked with
// the trailer's CRC32 and ISIZE
__global__ void member_check_kernel(const uint64_t* __restrict__ mem_trailer,
                                    const uint64_t* __restrict__ mem_len, uint32_t n_mem,
                                    const uint8_t* __restrict__ in,
                                    const uint32_t* __restrict__ mem_raw,
                                    uint32_t* __restrict__ mem_crc, int32_t* __restrict__ mem_status) {
  const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n_mem) return;
  const uint64_t t = mem_trailer[m];
  int32_t st = kOk;
  uint32_t crc = 0;
  if (t != kNoTrailer) {
    crc = ~(gf2_mulmod(x_pow_8n(mem_len[m]), 0xFFFFFFFFu) ^ mem_raw[m]);
    const uint32_t ecrc = in[t] | (in[t + 1] << 8) | ((uint32_t)in[t + 2] << 16) | ((uint32_t)in[t + 3] << 24);
    const uint32_t eisz = in[t + 4] | (in[t + 5] << 8) | ((uint32_t)in[t + 6] << 16) | ((uint32_t)in[t + 7] << 24);
    if ((uint32_t)mem_len[m] != eisz) st = kSizeMismatch;
    else if (crc != ecrc) st = kCrcMismatch;
  }
  mem_crc[m] = crc;
  mem_status[m] = st;
}

cudaError_t resolve_init(cudaStream_t stream) {
  crc_init_kernel<<<1, 256, 0, stream>>>();
  crc_shift_init_kernel<<<4 * kCrcLevels, 256, 0, stream>>>();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(crc_blocks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kCrcSmem);
}

cudaError_t launch_tail_literals(const PlacedChunk* placed, uint32_t n, const ChunkResult* results,
                                 const PagePool& pool, uint8_t* out, cudaStream_t stream) {
  if (!n) return cudaSuccess;
  tail_literals_kernel<<<n, 256, 0, stream>>>(placed, n, results, pool, out);
  return cudaGetLastError();
}

cudaError_t launch_tail_markers(const PlacedChunk* placed, const uint32_t* list, uint32_t n_list,
                                const ChunkResult* results, const PagePool& pool, uint8_t* out,
                                int sms, cudaStream_t stream) {
  if (!n_list) return cudaSuccess;
  const uint32_t grid = n_list < (uint32_t)(sms * 8) ? n_list : (uint32_t)(sms * 8);
  tail_markers_kernel<<<grid, 256, 0, stream>>>(placed, list, n_list, results, pool, out);
  return cudaGetLastError();
}

cudaError_t launch_body(const PlacedChunk* placed, const uint32_t* placed_of_chunk,
                        uint32_t n_pages, const ChunkResult* results, const PagePool& pool,
                        uint8_t* out, int sms, cudaStream_t stream) {
  if (!n_pages) return cudaSuccess;
  uint32_t blocks = n_pages < (uint32_t)(sms * 8) ? n_pages : (uint32_t)(sms * 8);
  body_kernel<<<blocks, 512, 0, stream>>>(placed, placed_of_chunk, n_pages, results, pool, out);
  return cudaGetLastError();
}

cudaError_t launch_crc(const CrcBlock* blocks, uint32_t n_blocks, const uint8_t* out,
                       const uint64_t* mem_end, uint32_t* mem_raw, const uint64_t* mem_trailer,
                       const uint64_t* mem_len, uint32_t n_mem, const uint8_t* in,
                       uint32_t* mem_crc, int32_t* mem_status, int sms, cudaStream_t stream) {
  if (n_blocks) {
    const uint32_t warps_per_cta = kCrcThreads / 32;
    const uint32_t need = (n_blocks + warps_per_cta - 1) / warps_per_cta;
    const uint32_t cap = (uint32_t)sms * kCrcCtasPerSm;
    const uint32_t grid = need < cap ? need : cap;
    crc_blocks_kernel<<<grid, kCrcThreads, kCrcSmem, stream>>>(blocks, n_blocks, out, mem_end,
                                                               mem_raw);
  }
  if (n_mem)
    member_check_kernel<<<(n_mem + 255) / 256, 256, 0, stream>>>(mem_trailer, mem_len, n_mem, in,
                                                                  mem_raw, mem_crc, mem_status);
  return cudaGetLastError();
}

}  // namespace gzgpu
