// finder.cuh -- launch interface of the block finder and chunk linking.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace gzgpu {

// n_sync (may be null) counts the sync starts found in fixed-Huffman data
cudaError_t launch_finder(const uint8_t* in, ChunkDesc* descs, const uint32_t* spec,
                          uint32_t n_spec, uint32_t* n_sync, cudaStream_t stream);
cudaError_t launch_link(ChunkDesc* descs, uint32_t n, uint32_t* work, uint32_t* n_work,
                        uint64_t slack_bits, cudaStream_t stream);

}  // namespace gzgpu
