// members.cuh -- launch interface of the member-location kernels.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace gzgpu {

struct StreamInfo {
  int32_t status;       // kOk, kNotGzip, kBadHeader, kTruncated
  uint32_t header_len;  // first member's header length
  uint32_t last_isize;  // last 4 bytes of the stream
  uint32_t first_btype; // BTYPE of the first block (0 stored, 1 fixed, 2 dynamic; 4 unknown)
};

struct ScanUnit {
  uint32_t stream;
  uint32_t pad;
  uint64_t begin, end;  // byte range relative to the stream start
};

struct MemberCand {
  uint64_t pos;         // relative to the stream start
  uint32_t stream;
  uint32_t header_len;  // 0 = malformed
  uint32_t prev_isize;
  uint32_t pad;
};

cudaError_t launch_stream_headers(const uint8_t* in, const uint64_t* s_off, const uint64_t* s_len,
                                  uint32_t n, StreamInfo* info, cudaStream_t stream);
cudaError_t launch_member_scan(const uint8_t* in, const ScanUnit* units, uint32_t n_units,
                               const uint64_t* s_off, const uint64_t* s_len,
                               const StreamInfo* info, MemberCand* cands, uint32_t* n_cands,
                               uint32_t cap, int sms, cudaStream_t stream);

}  // namespace gzgpu
