// finder.cu -- deflate block-boundary finder (K1) and chunk linking.
//
// One warp per speculative chunk searches [guess_bit, limit_bit) for the
// first block-start candidate (predicate and search in finder_core.cuh).
#include <cstdint>

#include "common.cuh"
#include "finder.cuh"
#include "finder_core.cuh"

namespace gzgpu {

__global__ void finder_kernel(const uint8_t* __restrict__ in, ChunkDesc* descs,
                              const uint32_t* __restrict__ spec, uint32_t n_spec) {
  const int lane = threadIdx.x & 31;
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= n_spec) return;
  ChunkDesc& d = descs[spec[w]];
  uint64_t lo = 0, hi = 0;
  bool have = warp_find_first(in, d.in_end, d.guess_bit, d.limit_bit, lane, lo, hi);
  if (lane == 0) {
    if (have) {
      d.lo_bit = lo;
      d.start_bit = hi;
      d.flags |= kChunkValid;
    } else {
      d.flags &= ~kChunkValid;
    }
  }
}

// stop_lo of each valid chunk = lo of the next valid chunk when that one is
// speculative (member starts end their predecessor at BFINAL instead);
// valid chunks are appended to the decode work list.
// A speculative start may be a phantom whose garbage code table never fails;
// such a chunk gives up `slack` bits past its stop and the chain walk
// re-decodes the gap from the confirmed boundary instead.
__global__ void link_kernel(ChunkDesc* descs, uint32_t n, uint32_t* work, uint32_t* n_work,
                            uint64_t slack) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ChunkDesc& d = descs[i];
  if (!(d.flags & kChunkValid)) return;
  uint64_t stop = kNoStop;
  for (uint32_t j = i + 1; j < n; j++) {
    uint32_t f = descs[j].flags;
    if (descs[j].stream != d.stream) break;
    if (f & kChunkMemberFirst) {
      // a member candidate (limit_bit = its header byte): a real one follows
      // the BFINAL block, a false one lies inside this member's data
      stop = descs[j].limit_bit * 8;
      break;
    }
    if (f & kChunkValid) {
      stop = descs[j].lo_bit;
      break;
    }
  }
  d.stop_lo = stop;
  d.abort_bit = (stop != kNoStop && !(d.flags & kChunkMemberFirst)) ? stop + slack : kNoStop;
  work[atomicAdd(n_work, 1u)] = i;
}

cudaError_t launch_finder(const uint8_t* in, ChunkDesc* descs, const uint32_t* spec,
                          uint32_t n_spec, cudaStream_t stream) {
  if (n_spec == 0) return cudaSuccess;
  const int warps = 8;
  uint32_t blocks = (n_spec + warps - 1) / warps;
  finder_kernel<<<blocks, 32 * warps, 0, stream>>>(in, descs, spec, n_spec);
  return cudaGetLastError();
}

cudaError_t launch_link(ChunkDesc* descs, uint32_t n, uint32_t* work, uint32_t* n_work,
                        uint64_t slack_bits, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  link_kernel<<<(n + 255) / 256, 256, 0, stream>>>(descs, n, work, n_work, slack_bits);
  return cudaGetLastError();
}

}  // namespace gzgpu
