// finder.cu -- deflate block-boundary finder (K1) and chunk linking.
//
// Each speculative chunk searches [guess_bit, limit_bit) for its first
// block-start candidate (predicate and search in finder_core.cuh) with the
// warps of one CTA.
#include <cstdint>

#include "common.cuh"
#include "finder.cuh"
#include "finder_core.cuh"

namespace gzgpu {

// One CTA per speculative chunk.  Its warps take the 1024-bit windows of
// [guess_bit, limit_bit) round-robin, each window searched for its first
// candidate (by start bit, so windows partition the candidates); a warp stops
// as soon as a lower window has a hit, so the work is about the distance to
// the first candidate, split over the CTA's warps.  Stored candidates must
// also pass start_ok (a stored or dynamic block right after them).
constexpr int kFinderWarps = 2;
constexpr uint64_t kFinderWindow = 1024 * kFindGroup;  // bits a warp takes at a time

// Stored block starts, searched first for every speculative chunk: the first
// one (by byte offset, hence by start bit) in [guess_bit, limit_bit) whose
// successor passes stored_successor_ok becomes the chunk's start, and the
// sync search and the block finder skip the chunk.  The successor check is
// a heuristic: a false start needs two LEN/NLEN matches in a row, or a
// LEN/NLEN match and a valid dynamic header, which is rare but possible.
// Correctness does not rest on it: a false start only decodes garbage that
// no predecessor hands over to, and the host chain walk repairs past it.
// The pass runs before the sync search because the raw bytes of stored
// blocks (text, runs) walk as fixed-Huffman codes and would give false sync
// starts.  One CTA of kStoredThreads per chunk, scanning that many byte
// offsets a round.
constexpr int kStoredThreads = 256;

__global__ void __launch_bounds__(kStoredThreads)
    stored_kernel(const uint8_t* __restrict__ in, ChunkDesc* descs,
                  const uint32_t* __restrict__ spec, uint32_t n_spec) {
  __shared__ unsigned long long s_first;
  unsigned long long* s_off = &s_first;
  if (blockIdx.x >= n_spec) return;
  ChunkDesc& d = descs[spec[blockIdx.x]];
  if (d.flags & kChunkValid) return;
  const uint64_t from = d.guess_bit, to = d.limit_bit, nbytes = d.in_end;
  if (threadIdx.x == 0) *s_off = ~0ull;
  __syncthreads();
  const uint64_t until = nbytes >= 5 ? min((to + 7) / 8, nbytes - 4) : 0;
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  // each thread screens 4 consecutive byte offsets a round for LEN == ~NLEN
  for (uint64_t base = max((from + 3 + 7) / 8, (uint64_t)2); base < until; base += 4 * blockDim.x) {
    const uint64_t ob = base + 4 * (uint64_t)threadIdx.x;
    uint32_t m = 0;
    if (ob < until) {
      m = stored_filter4(bits64_at(in32, ob * 8));
      if (ob + 4 > until) m &= (1u << (until - ob)) - 1;
    }
    while (m) {
      const uint64_t off = ob + (uint64_t)(__ffs(m) - 1);
      m &= m - 1;
      uint64_t lo = 0, hi = 0;
      if (stored_candidate(in, nbytes, off, from, to, to, lo, hi) &&
          stored_successor_ok(in, nbytes, off + 4 + (in[off] | (in[off + 1] << 8)))) {
        atomicMin(s_off, (unsigned long long)off);
        break;
      }
    }
    __syncthreads();
    const bool found = *s_off != ~0ull;
    __syncthreads();  // every thread has read it before the next round writes
    if (found) break;
  }
  if (threadIdx.x == 0 && *s_off != ~0ull) {
    uint64_t lo = 0, hi = 0;
    stored_candidate(in, nbytes, *s_off, from, to, to, lo, hi);
    d.lo_bit = lo;
    d.start_bit = hi;
    d.flags |= kChunkValid;
    d.est_ratio = 1.f;
  }
}

// The precode leaf count of 4 code-length codes (12 bits) for every value,
// built at compile time and read through the L1 cache: a CTA needs no
// shared copy, so more small CTAs fit on an SM.
struct LeafLut {
  uint16_t v[4096];
  constexpr LeafLut() : v() {
    for (int i = 0; i < 4096; i++) {
      uint32_t sum = 0;
      for (int k = 0; k < 4; k++) {
        const uint32_t L = (i >> (3 * k)) & 7;
        sum += L ? 1u << (7 - L) : 0u;
      }
      v[i] = (uint16_t)sum;
    }
  }
};
__device__ const LeafLut d_leaf_lut = LeafLut();

__global__ void __launch_bounds__(32 * kFinderWarps)
    finder_kernel(const uint8_t* __restrict__ in, ChunkDesc* descs,
                  const uint32_t* __restrict__ spec, uint32_t n_spec) {
  __shared__ unsigned long long best_win;
  __shared__ uint64_t hit_lo[kFinderWarps], hit_hi[kFinderWarps], hit_win[kFinderWarps];
  __shared__ FinderLists lists[kFinderWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (blockIdx.x >= n_spec) return;
  ChunkDesc& d = descs[spec[blockIdx.x]];
  if (d.flags & kChunkValid) return;  // a stored or sync start was found first
  const uint16_t* leaf_lut = d_leaf_lut.v;
  const uint64_t from = d.guess_bit, to = d.limit_bit, nbytes = d.in_end;
  if (threadIdx.x == 0) best_win = ~0ull;
  if (lane == 0) hit_win[warp] = ~0ull;
  __syncthreads();
  const uint64_t n_win = to > from ? (to - from + kFinderWindow - 1) / kFinderWindow : 0;
  for (uint64_t k = warp; k < n_win; k += kFinderWarps) {
    if (k > *(volatile unsigned long long*)&best_win) break;
    const uint64_t w0 = from + k * kFinderWindow;
    const uint64_t w1 = min(w0 + kFinderWindow, to);
    uint64_t lo = 0, hi = 0, s0 = w0;
    bool hit = false;
    // stored candidates: the stored-start pass before this kernel took the
    // first that could start this range, so only dynamic ones are left
    while (s0 < w1 &&
           warp_find_first(in, nbytes, s0, w1, to, lane, lo, hi, leaf_lut, &lists[warp], true)) {
      if (start_ok(in, nbytes, hi)) {
        hit = true;
        break;
      }
      s0 = lo + 1;  // a stored match without a plausible successor
    }
    if (hit) {
      if (lane == 0) {
        hit_lo[warp] = lo;
        hit_hi[warp] = hi;
        hit_win[warp] = k;
        atomicMin(&best_win, (unsigned long long)k);
      }
      break;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t bw = ~0ull;
    int bwarp = -1;
    for (int i = 0; i < kFinderWarps; i++)
      if (hit_win[i] < bw) {
        bw = hit_win[i];
        bwarp = i;
      }
    if (bwarp >= 0) {
      d.lo_bit = hit_lo[bwarp];
      d.start_bit = hit_hi[bwarp];
      d.flags |= kChunkValid;
      // BTYPE at the start: 2 = dynamic (estimate from its code lengths), 0 = stored
      const uint32_t bt = (uint32_t)(peek_bits(in, nbytes, d.start_bit, 3) >> 1);
      d.est_ratio = bt == 2 ? dyn_header_ratio(in, nbytes, d.start_bit) : 1.f;
    } else {
      d.flags &= ~kChunkValid;
    }
  }
}

// Sync starts in fixed-Huffman data (finder_core.cuh fixed_walk), searched
// for every speculative chunk before the block finder, which then skips the
// chunks that have one.  One CTA of kSyncOffsets threads per chunk; the walk
// must end inside the chunk's range and the input.
__global__ void __launch_bounds__(kSyncOffsets)
    sync_kernel(const uint8_t* __restrict__ in, ChunkDesc* descs, const uint32_t* __restrict__ spec,
                uint32_t n_spec, uint32_t* n_sync) {
  __shared__ uint32_t sync_words[kSyncWords];
  __shared__ uint64_t sync_end[kSyncOffsets];
  if (blockIdx.x >= n_spec) return;
  ChunkDesc& d = descs[spec[blockIdx.x]];
  if (d.flags & kChunkValid) return;
  const uint64_t from = d.guess_bit, to = d.limit_bit, nbytes = d.in_end;
  const uint64_t target = from + kSyncOffsets + kSyncSpan;
  if (target + 64 > to || target + 128 > nbytes * 8) return;
  const uint64_t wbase = from >> 5;
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  for (uint32_t i = threadIdx.x; i < kSyncWords; i += blockDim.x) sync_words[i] = in32[wbase + i];
  __syncthreads();
  if (threadIdx.x < kSyncOffsets)
    sync_end[threadIdx.x] = fixed_walk(sync_words, wbase, from + threadIdx.x, target);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t best = kSyncFail;
    uint32_t best_n = 1;
    for (uint32_t i = 0; i < kSyncOffsets; i++) {
      const uint64_t v = sync_end[i];
      if (v == kSyncFail) continue;
      uint32_t c = 0;
      for (uint32_t j = 0; j < kSyncOffsets; j++) c += sync_end[j] == v;
      if (c > best_n || (c == best_n && best != kSyncFail && v < best)) {
        best = v;
        best_n = c;
      }
    }
    if (best != kSyncFail) {
      d.lo_bit = d.start_bit = best;
      d.flags |= kChunkValid | kChunkSync;
      if (n_sync) atomicAdd(n_sync, 1u);
    }
  }
}

// stop_lo of each valid chunk = lo of the next valid chunk when that one is
// speculative (member starts end their predecessor at BFINAL instead);
// valid chunks are appended to the decode work list.
// A speculative start may be a phantom whose garbage code table never fails;
// such a chunk gives up `slack` bits past its stop and the chain walk
// re-decodes the gap from the confirmed boundary instead.
// Decode cost of a linked chunk.  The decoder's time follows its compressed
// bits (one step per 32 bits) plus its copy work, which follows the output:
// measured per 64 KiB chunk of the 1 GiB mixed stream, about 12.5 ms at 1
// output byte per input byte (near-incompressible literals), 16 ms at 2.9
// (text) and 29 ms at 13.6 (byte runs), and 0.6 ms for stored data.  So the
// cost is the compressed bytes times (1 + 0.2 x the output-per-input estimate
// of the dynamic header a chunk starts in), and a twentieth of that for a
// stored start: the decode cost per compressed byte of the data a chunk
// start begins in.
__device__ float cost_factor(const uint8_t* __restrict__ in, const ChunkDesc& d) {
  float r = d.est_ratio;
  if (!(r > 0.f)) {
    // member starts and sync starts carry no finder estimate: take it from
    // the header of the block they start in
    const uint64_t hdr = (d.flags & kChunkSync) ? d.table_bit : d.start_bit;
    const uint32_t bt = hdr ? (uint32_t)(peek_bits(in, d.in_end, hdr, 3) >> 1) : 1u;
    if (bt == 0) return 0.05f;
    if (bt == 2) r = dyn_header_ratio(in, d.in_end, hdr);
    if (!(r > 0.f)) r = 2.f;  // fixed-Huffman data: about 2 bytes per input byte
  } else if (r == 1.f && (peek_bits(in, d.in_end, d.start_bit, 3) >> 1) == 0) {
    return 0.05f;  // a stored start
  }
  return 1.f + 0.2f * r;
}

// A chunk's cost is its compressed bytes times the larger of the factors of
// its own start and of its successor's, which shows the data at its far end:
// a chunk that starts in stored data and runs into dense text or byte runs
// is as costly as that data.
__device__ float chunk_cost(const uint8_t* __restrict__ in, const ChunkDesc* descs,
                            const ChunkDesc& d, uint64_t stop, uint32_t next) {
  const uint64_t nbits = d.in_end * 8;
  uint64_t end = stop != kNoStop ? stop : nbits;
  if (end > nbits) end = nbits;
  const float span = end > d.start_bit ? (float)(end - d.start_bit) * 0.125f : 0.f;
  float f = cost_factor(in, d);
  if (next != kNoChunk && !(descs[next].flags & kChunkMemberFirst))
    f = fmaxf(f, cost_factor(in, descs[next]));
  return f * span;
}

__global__ void link_kernel(const uint8_t* __restrict__ in, ChunkDesc* descs, uint32_t n,
                            uint32_t* work, uint32_t* n_work, float* cost, uint64_t slack) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ChunkDesc& d = descs[i];
  if (!(d.flags & kChunkValid)) return;
  uint64_t stop = kNoStop;
  uint32_t next = kNoChunk;
  for (uint32_t j = i + 1; j < n; j++) {
    uint32_t f = descs[j].flags;
    if (descs[j].stream != d.stream) break;
    if (f & kChunkMemberFirst) {
      // a member candidate (limit_bit = its header byte): a real one follows
      // the BFINAL block, a false one lies inside this member's data
      stop = descs[j].limit_bit * 8;
      next = j;
      break;
    }
    if (f & kChunkValid) {
      stop = descs[j].lo_bit;
      next = j;
      break;
    }
  }
  d.stop_lo = stop;
  d.next = next;
  // A sync start whose table or alignment is wrong decodes garbage that a
  // complete code never rejects: it may run at most its own length (at least
  // kSyncMinSlack) past its stop.  A real one stops at its successor, or goes
  // by phantom successors mid-block to the one after (inflate.cu).
  uint64_t s = slack;
  if ((d.flags & kChunkSync) && stop != kNoStop && stop > d.start_bit)
    s = min(slack, max(stop - d.start_bit, (uint64_t)kSyncMinSlack));
  d.abort_bit = (stop != kNoStop && !(d.flags & kChunkMemberFirst)) ? stop + s : kNoStop;
  if (cost) cost[i] = chunk_cost(in, descs, d, stop, next);
  else work[atomicAdd(n_work, 1u)] = i;
}

// The decode work list in descending cost (longest processing time first),
// so that the persistent decoder starts the longest chunks first and the
// short ones fill in at the end.  One CTA: a histogram over half-octave cost
// buckets, a scan, and a scatter (order inside a bucket is arbitrary).
constexpr int kCostBuckets = 64;
__global__ void __launch_bounds__(1024)
    order_kernel(const ChunkDesc* __restrict__ descs, const float* __restrict__ cost, uint32_t n,
                 uint32_t* work, uint32_t* n_work) {
  __shared__ uint32_t hist[kCostBuckets], base[kCostBuckets];
  if (threadIdx.x < kCostBuckets) hist[threadIdx.x] = 0;
  __syncthreads();
  auto bucket = [&](uint32_t i) {
    const float c = fmaxf(cost[i], 0.f) + 1.f;
    const int b = (int)(2.f * __log2f(c));
    return kCostBuckets - 1 - min(max(b, 0), kCostBuckets - 1);  // costliest first
  };
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
    if (descs[i].flags & kChunkValid) atomicAdd(&hist[bucket(i)], 1u);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t a = 0;
    for (int b = 0; b < kCostBuckets; b++) {
      base[b] = a;
      a += hist[b];
    }
    *n_work = a;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
    if (descs[i].flags & kChunkValid) work[atomicAdd(&base[bucket(i)], 1u)] = i;
}

cudaError_t launch_finder(const uint8_t* in, ChunkDesc* descs, const uint32_t* spec,
                          uint32_t n_spec, uint32_t* n_sync, cudaStream_t stream) {
  if (n_spec == 0) return cudaSuccess;
  // Stored starts first (a byte scan), then the fixed-code sync search: it
  // costs a fraction of a full scan, which a fixed-Huffman partition (no
  // block header to find) would need, and it fails within a few dozen
  // symbols on other data.
  stored_kernel<<<n_spec, kStoredThreads, 0, stream>>>(in, descs, spec, n_spec);
  sync_kernel<<<n_spec, kSyncOffsets, 0, stream>>>(in, descs, spec, n_spec, n_sync);
  finder_kernel<<<n_spec, 32 * kFinderWarps, 0, stream>>>(in, descs, spec, n_spec);
  return cudaGetLastError();
}

cudaError_t launch_link(const uint8_t* in, ChunkDesc* descs, uint32_t n, uint32_t* work,
                        uint32_t* n_work, float* cost, uint64_t slack_bits, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  link_kernel<<<(n + 255) / 256, 256, 0, stream>>>(in, descs, n, work, n_work, cost, slack_bits);
  if (cost) order_kernel<<<1, 1024, 0, stream>>>(descs, cost, n, work, n_work);
  return cudaGetLastError();
}

}  // namespace gzgpu
