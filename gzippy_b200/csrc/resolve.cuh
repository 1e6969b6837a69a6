// resolve.cuh -- launch interface of window propagation, marker resolution and CRC.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace gzgpu {

cudaError_t resolve_init(cudaStream_t stream);
cudaError_t launch_tail_literals(const PlacedChunk* placed, uint32_t n, const ChunkResult* results,
                                 const PagePool& pool, uint8_t* out, cudaStream_t stream);
cudaError_t launch_tail_markers(const PlacedChunk* placed, const uint32_t* list, uint32_t n_list,
                                const ChunkResult* results, const PagePool& pool, uint8_t* out,
                                int sms, cudaStream_t stream);
cudaError_t launch_body(const PlacedChunk* placed, const uint32_t* placed_of_chunk,
                        uint32_t n_pages, const ChunkResult* results, const PagePool& pool,
                        uint8_t* out, int sms, cudaStream_t stream);
// CRC: one warp per block of up to kCrcBlock bytes, 32 lane slices of
// kCrcSlice bytes each
constexpr uint32_t kCrcBlock = 32768;
constexpr uint32_t kCrcSlice = kCrcBlock / 32;
constexpr int kCrcThreads = 512;
constexpr int kCrcCtasPerSm = 4;
constexpr int kCrcLevels = 5;  // log2(32 slices)
// shared memory: 32 lane copies of the byte table, shift tables
constexpr size_t kCrcSmem = 256 * 32 * 4 + kCrcLevels * 4 * 256 * 4;

// mem_end[m]: output offset just past member m; mem_raw[m]: its CRC register
// accumulator (zeroed before the launch); then each member's CRC and status
cudaError_t launch_crc(const CrcBlock* blocks, uint32_t n_blocks, const uint8_t* out,
                       const uint64_t* mem_end, uint32_t* mem_raw, const uint64_t* mem_trailer,
                       const uint64_t* mem_len, uint32_t n_mem, const uint8_t* in,
                       uint32_t* mem_crc, int32_t* mem_status, int sms, cudaStream_t stream);

}  // namespace gzgpu
