// inflate.cuh -- launch interface of the chunk inflate kernel.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace gzgpu {

constexpr int kDecodeWarps = 1;  // warps (= chunks in flight) per CTA
constexpr int kDistBits = 8;     // distance LUT index bits

template <int LB>
size_t inflate_smem_bytes();
template <int LB>
int inflate_blocks_per_sm();
template <int LB>
cudaError_t launch_inflate(const uint8_t* in, const ChunkDesc* descs, ChunkResult* results,
                           const uint32_t* work, const uint32_t* n_work, uint32_t* work_counter,
                           const PagePool& pool, int blocks, cudaStream_t stream);

}  // namespace gzgpu
