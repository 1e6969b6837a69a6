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
cudaError_t launch_crc(const CrcBlock* blocks, uint32_t n_blocks, const uint8_t* out,
                       uint32_t* block_crcs, const uint32_t* mem_block_begin,
                       const uint64_t* mem_trailer, const uint64_t* mem_len, uint32_t n_mem,
                       const uint8_t* in, uint32_t* mem_crc, int32_t* mem_status, int sms,
                       cudaStream_t stream);

}  // namespace gzgpu
