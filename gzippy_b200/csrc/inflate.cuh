// inflate.cuh -- launch interface of the chunk inflate kernels.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace gzgpu {

constexpr int kRingWarps = 1;      // ring kernel: warps per CTA (64 KB ring each)
constexpr int kPageWarps = 8;      // page kernel: warps per CTA (tables only)
constexpr int kDistBits = 8;       // distance LUT index bits

template <int LB>
size_t inflate_smem_bytes(bool ring);
// page kernel: `ctas` (3 or 4) CTAs of kPageWarps warps per SM; registers are
// sized for that many (80 or 64 per thread)
template <int LB>
int inflate_blocks_per_sm(bool ring, int ctas);
template <int LB>
// sync: the job has sync starts (selects the kernel variant that handles them)
cudaError_t launch_inflate(bool ring, int ctas, bool sync, const uint8_t* in, ChunkDesc* descs,
                           ChunkResult* results, const uint32_t* work, const uint32_t* n_work,
                           uint32_t* work_counter, const PagePool& pool, int blocks,
                           cudaStream_t stream);
// sync starts inside dynamic blocks for the listed pieces left without a start
cudaError_t launch_dyn_sync(const uint8_t* in, ChunkDesc* descs, const uint32_t* pieces, uint32_t n,
                            uint32_t* n_sync, cudaStream_t stream);

}  // namespace gzgpu
