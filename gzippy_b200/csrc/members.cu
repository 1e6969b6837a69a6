// members.cu -- gzip member location on the device.
//
// stream_header_kernel: per stream, the magic check (non-gzip -> kNotGzip,
//   src/lib.rs:50-52) and the first member's header length (RFC 1952,
//   gzip_format.rs read_header :47-133).
// member_scan_kernel: every byte position of every stream is tested like
//   scan_member_boundaries_fast (src/decompress/bgzf.rs:2090-2230): bytes
//   1f 8b 08, FLG & 0xE0 == 0, pos >= 4, the preceding ISIZE in (0, 1 GiB],
//   pos past the first header and pos + 10 < stream length; plus the header
//   plausibility of is_likely_multi_member (src/decompress/format.rs:92-125:
//   MTIME, XFL, OS), which removes nearly every false hit in compressed data.
//   A real member that fails it is still found by the host chain walk.
//   Each hit's header is parsed (parse_gzip_header :2047) for its deflate
//   start.
#include <cstdint>

#include "common.cuh"
#include "members.cuh"

namespace gzgpu {

// header length of the member at `p` (absolute), bounded by `end`;
// returns 0 on a malformed or truncated header.
__device__ uint64_t parse_header(const uint8_t* in, uint64_t p, uint64_t end) {
  if (end < p + 10) return 0;
  if (in[p] != 0x1f || in[p + 1] != 0x8b || in[p + 2] != 8) return 0;
  uint8_t flg = in[p + 3];
  if (flg & 0xE0) return 0;
  uint64_t o = p + 10;
  if (flg & 4) {
    if (o + 2 > end) return 0;
    uint64_t xlen = in[o] | (in[o + 1] << 8);
    o += 2 + xlen;
    if (o > end) return 0;
  }
  for (int f = 8; f <= 16; f <<= 1) {
    if (flg & f) {
      uint64_t lim = o + 65536;  // bounded walk
      while (o < end && o < lim && in[o]) o++;
      if (o >= end || o >= lim) return 0;
      o++;
    }
  }
  if (flg & 2) {
    o += 2;
    if (o > end) return 0;
  }
  return o - p;
}

__global__ void stream_header_kernel(const uint8_t* __restrict__ in,
                                     const uint64_t* __restrict__ s_off,
                                     const uint64_t* __restrict__ s_len, uint32_t n,
                                     StreamInfo* info) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint64_t p = s_off[s], len = s_len[s];
  StreamInfo si{};
  if (len < 2 || in[p] != 0x1f || in[p + 1] != 0x8b) {
    si.status = kNotGzip;
  } else {
    uint64_t h = parse_header(in, p, p + len);
    if (h == 0) {
      si.status = (len < 10 || in[p + 2] == 8) ? kTruncated : kBadHeader;
      if (len >= 10 && in[p + 2] == 8 && (in[p + 3] & 0xE0)) si.status = kBadHeader;
    } else {
      si.status = kOk;
      si.header_len = (uint32_t)h;
    }
  }
  si.first_btype = 4;
  if (si.status == kOk && si.header_len < len) si.first_btype = (in[p + si.header_len] >> 1) & 3;
  if (len >= 4) {
    const uint8_t* t = in + p + len - 4;
    si.last_isize = t[0] | (t[1] << 8) | ((uint32_t)t[2] << 16) | ((uint32_t)t[3] << 24);
  }
  info[s] = si;
}

// bit 7 of each byte of the result is set exactly where w's byte is zero
__device__ __forceinline__ uint32_t zero_bytes(uint32_t w) {
  const uint32_t t = (w & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
  return ~(t | w | 0x7F7F7F7Fu);
}

// grid-stride over scan units (stream, byte range); each thread screens 16
// aligned bytes at a time for the 0x1f of the magic with word operations
// and tests only the positions that have one
__global__ void member_scan_kernel(const uint8_t* __restrict__ in, const ScanUnit* __restrict__ units,
                                   uint32_t n_units, const uint64_t* __restrict__ s_off,
                                   const uint64_t* __restrict__ s_len,
                                   const StreamInfo* __restrict__ info, MemberCand* cands,
                                   uint32_t* n_cands, uint32_t cap) {
  for (uint32_t u = blockIdx.x; u < n_units; u += gridDim.x) {
    const ScanUnit su = units[u];
    const StreamInfo si = info[su.stream];
    if (si.status != kOk) continue;
    const uint64_t base = s_off[su.stream], len = s_len[su.stream];
    const uint64_t lo = su.begin > (uint64_t)si.header_len + 1 ? su.begin : si.header_len + 1;
    for (uint64_t a = ((base + lo) & ~15ull) + 16 * (uint64_t)threadIdx.x; a < base + su.end;
         a += 16 * (uint64_t)blockDim.x) {
      const uint4 v = *reinterpret_cast<const uint4*>(in + a);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        uint32_t m = zero_bytes(w[k] ^ 0x1F1F1F1Fu);
        while (m) {
          const int j = (__ffs(m) - 1) >> 3;
          m &= m - 1;
          const uint64_t pos = a + 4 * k + j - base;
          if (pos < lo || pos >= su.end) continue;
          if (pos + 10 >= len || pos < 4) continue;
          const uint8_t* q = in + base + pos;
          if (q[0] != 0x1f || q[1] != 0x8b || q[2] != 8 || (q[3] & 0xE0)) continue;
          const uint32_t isz =
              q[-4] | (q[-3] << 8) | ((uint32_t)q[-2] << 16) | ((uint32_t)q[-1] << 24);
          if (isz == 0 || isz > (1u << 30)) continue;
          // header plausibility of is_likely_multi_member (format.rs:92-125):
          // MTIME 0 or <= 4102444800, XFL in {0, 2, 4}, OS <= 13 or 255
          const uint32_t mtime =
              q[4] | (q[5] << 8) | ((uint32_t)q[6] << 16) | ((uint32_t)q[7] << 24);
          if (mtime > 4102444800u) continue;
          if (q[8] != 0 && q[8] != 2 && q[8] != 4) continue;
          if (q[9] > 13 && q[9] != 255) continue;
          const uint32_t kk = atomicAdd(n_cands, 1u);
          if (kk < cap) {
            MemberCand c;
            c.stream = su.stream;
            c.pos = pos;
            c.header_len = (uint32_t)parse_header(in, base + pos, base + len);
            c.prev_isize = isz;
            cands[kk] = c;
          }
        }
      }
    }
  }
}

cudaError_t launch_stream_headers(const uint8_t* in, const uint64_t* s_off, const uint64_t* s_len,
                                  uint32_t n, StreamInfo* info, cudaStream_t stream) {
  if (!n) return cudaSuccess;
  stream_header_kernel<<<(n + 127) / 128, 128, 0, stream>>>(in, s_off, s_len, n, info);
  return cudaGetLastError();
}

cudaError_t launch_member_scan(const uint8_t* in, const ScanUnit* units, uint32_t n_units,
                               const uint64_t* s_off, const uint64_t* s_len,
                               const StreamInfo* info, MemberCand* cands, uint32_t* n_cands,
                               uint32_t cap, int sms, cudaStream_t stream) {
  if (!n_units) return cudaSuccess;
  uint32_t grid = n_units < (uint32_t)(sms * 16) ? n_units : (uint32_t)(sms * 16);
  member_scan_kernel<<<grid, 512, 0, stream>>>(in, units, n_units, s_off, s_len, info, cands,
                                                n_cands, cap);
  return cudaGetLastError();
}

}  // namespace gzgpu
