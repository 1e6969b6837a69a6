// finder.cuh -- launch interface of the block finder and chunk linking.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace gzgpu {

// n_sync (may be null) counts the sync starts found in fixed-Huffman data
cudaError_t launch_finder(const uint8_t* in, ChunkDesc* descs, const uint32_t* spec,
                          uint32_t n_spec, uint32_t* n_sync, cudaStream_t stream);
// links every valid chunk to its successor and writes the decode work list:
// in descending decode cost when `cost` (n floats of scratch) is given, else
// in no particular order
cudaError_t launch_link(const uint8_t* in, ChunkDesc* descs, uint32_t n, uint32_t* work,
                        uint32_t* n_work, float* cost, uint64_t slack_bits, cudaStream_t stream);

}  // namespace gzgpu
