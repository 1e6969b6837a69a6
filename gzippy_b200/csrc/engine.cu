// engine.cu -- host driver of the B200 gzip decode pipeline and the C ABI.
//
// One job decodes a set of streams that sit back to back in one device
// input buffer.  Stages (device unless noted):
//   1. stream headers + member scan            (members.cu)
//   2. chunk grid per member                   (host: partitions of chunk_bytes)
//   3. block finder + link                     (finder.cu)
//   4. persistent inflate over the work list   (inflate.cu)
//   5. chain walk                              (host: accept / repair, as the
//      reference's consumer_loop, chunk_fetcher.rs:855; repairs re-enter 4)
//   6. tails, window chain, bodies, CRC        (resolve.cu)
// The plain path (gzgpu_decompress) runs one stream per job; the batched
// path runs all of a batch's streams in one job, so every stage is one launch
// for the whole batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/gzgpu.h"
#include "common.cuh"
#include "finder.cuh"
#include "inflate.cuh"
#include "members.cuh"
#include "resolve.cuh"
#include "stage.h"

using namespace gzgpu;

namespace {

// Device buffer that grows in stream order on its context's stream
// (cudaMallocAsync / cudaFreeAsync): growing one context's buffers does not
// synchronize the device, so contexts on other threads keep running.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaStream_t st = nullptr;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
    size_t want = n + n / 4 + 4096;
    cudaError_t e = cudaMallocAsync(&p, want, st);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  // grow to at least n bytes, keeping the first `keep` bytes
  cudaError_t grow_keep(size_t n, size_t keep) {
    if (n <= cap) return cudaSuccess;
    void* q = nullptr;
    const size_t want = n + n / 4 + 4096;
    cudaError_t e = cudaMallocAsync(&q, want, st);
    if (e != cudaSuccess) return e;
    if (p && keep) e = cudaMemcpyAsync(q, p, std::min(keep, cap), cudaMemcpyDeviceToDevice, st);
    if (p) cudaFreeAsync(p, st);
    p = q;
    cap = want;
    return e;
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

struct HostPinned {
  void* p = nullptr;
  size_t cap = 0;
  bool ensure(size_t n) {
    if (n <= cap) return true;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = n + n / 4 + 4096;
    if (cudaMallocHost(&p, want) != cudaSuccess) return false;
    cap = want;
    return true;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

struct StreamSpec {
  uint64_t off, len;  // byte range in the device input buffer
};

struct StreamOut {
  int status = kOk;
  uint64_t out_off = 0, out_len = 0;
};

struct MemberPlan {
  uint32_t order_begin, order_end;  // range in the stream's chunk order
  uint64_t trailer;                 // absolute input byte of the CRC32/ISIZE trailer
  uint64_t out_len;
};

// chain walk state (host) of one segment of a stream: the members from one
// planned member start up to the next planned start (`mend`), or the whole
// stream (`last`).  Segments of a multi-member stream are walked
// independently, so their repairs share decode passes; a segment must end
// exactly at `mend`, else its stream is walked again as one segment.
struct Walker {
  uint32_t stream;
  uint32_t c0, c1;          // grid chunk ids of this segment [c0, c1)
  uint32_t j;               // next grid chunk to consider
  uint64_t mpos;            // next member header, relative to the stream
  uint64_t mend = 0;        // planned start of the next segment (relative)
  bool last = true;         // segment runs to the end of the stream
  bool handoff_bad = false; // ended somewhere other than `mend`
  uint32_t member = 0;
  int32_t cur = -1;         // chunk being walked
  bool done = false;
  int status = kOk;
  std::vector<uint32_t> order;
  std::vector<MemberPlan> members;
  uint32_t member_order_begin = 0;
  int32_t pending = -1;     // repair chunk id awaiting decode (walk suspended)
  // Optimistic repairs: a repair is assumed to end exactly at the next
  // candidate's start and the walk goes on; `cp` restores the walk if the
  // decoded repair says otherwise.
  struct Checkpoint {
    size_t order_size, members_size;
    uint32_t j, member, member_order_begin;
    uint64_t mpos;
  };
  struct Assumption {
    uint32_t repair;
    uint64_t lo, hi;  // the next chunk's acceptable start range
    bool sync;        // the next chunk is a sync start (taken over mid-block)
    Checkpoint cp;
  };
  std::vector<Assumption> assumed;
};

const char* kErrStr[] = {"ok",
                         "not a gzip stream",
                         "invalid gzip header",
                         "invalid deflate data",
                         "CRC32 mismatch",
                         "ISIZE mismatch",
                         "output buffer too small",
                         "CUDA device error",
                         "timed out",
                         "truncated input",
                         "device page pool exhausted",
                         "chunk not decoded",
                         "invalid argument",
                         "speculative chunk overshot its stop",
                         "output exceeds the 4 MiB limit of the no-allocation entry point",
                         "request exceeds the server's device-memory budget",
                         "request still pending"};

}  // namespace

struct gzgpu_ctx {
  std::mutex mu;
  int dev = 0, sms = 148;
  cudaStream_t st = nullptr;
  size_t chunk_bytes = 0;
  int lut_bits = 10;
  bool autotune = false;
  bool ring = false;  // history layout of the inflate kernel (false = pages)
  int ctas_per_sm = 3;  // page kernel CTAs per SM (3 or 4)
  uint32_t decoder_mode = 3;  // PagePool::serial: Huffman block decoder (3: chosen per block)
  bool fine_split = false;  // output-estimate pieces + dynamic-block sync starts
  bool high_priority = false;  // stream at the device's greatest priority
  bool lpt = true;             // decode work list longest-first (else in stream order)
  bool job_raw = false;        // the job's streams are raw DEFLATE (no gzip framing)
  bool job_sync = true;     // the running job has sync starts (decoder variant)
  int decode_blocks = 0;
  cudaEvent_t ev[12];
  cudaEvent_t stage_ev[2];  // last DMA of each pinned staging slot
  gzgpu_stats stats{};
  bool crc_ready = false;

  DevBuf in, out, s_off, s_len, info, units, cands, counters, descs, results, spec, work, cost;
  DevBuf pages, owner, seq, placed, placed_of, list, cblocks, mend, mraw, mtrail, mlen, mcrc,
      mstatus;
  // seek-index builds: the decoder's block log, the checkpoint interval and
  // the serialized index of the last job (gzgpu_build_index)
  DevBuf blk_log;
  uint32_t blk_cap = 0, blk_need = 0;
  bool job_index = false;
  uint64_t index_interval = 0;
  int index_status = 0;
  std::vector<uint8_t> index_bytes;
  HostPinned h_stage;
  std::vector<DevBuf*> all_bufs() {
    return {&in,     &out,   &s_off,   &s_len,  &info,   &units,   &cands,  &counters, &descs,
            &results, &spec, &work,    &pages,  &owner,  &seq,     &placed, &placed_of, &list,
            &cblocks, &mend,  &mraw,   &mtrail, &mlen,    &mcrc,   &mstatus, &blk_log,
            &cost};
  }
  const uint8_t* cur_in = nullptr;  // input buffer of the running job
  uint8_t* user_out = nullptr;       // caller device output (device-resident API)
  size_t user_cap = 0;
  uint8_t* cur_out = nullptr;        // output buffer the job resolved into

  int check(cudaError_t e) {
    if (e != cudaSuccess) {
      fprintf(stderr, "gzgpu: CUDA error %s\n", cudaGetErrorString(e));
      return kDeviceError;
    }
    return kOk;
  }

  cudaError_t launch_decode(uint32_t* d_work_count) {
    PagePool pool{pages.as<uint16_t>(), owner.as<uint32_t>(), seq.as<uint32_t>(),
                  counters.as<uint32_t>() + 2, (uint32_t)(pages.cap / (kPageEntries * 2))};
    pool.cap = (uint32_t)std::min<uint64_t>(pool.cap, std::min(owner.cap, seq.cap) / 4);
    pool.serial = decoder_mode;
    if (job_index) {
      pool.blocks = blk_log.as<BlockRec>();
      pool.n_blocks = counters.as<uint32_t>() + 8;
      pool.blocks_cap = blk_cap;
    }
    cudaError_t e = cudaMemsetAsync(counters.as<uint32_t>() + 3, 0, 4, st);
    if (e != cudaSuccess) return e;
    stats.kernel_launches++;
    stats.decode_passes++;
    switch (lut_bits) {
      case 11:
        return launch_inflate<11>(ring, ctas_per_sm, job_sync, cur_in, descs.as<ChunkDesc>(), results.as<ChunkResult>(),
                                  work.as<uint32_t>(), d_work_count, counters.as<uint32_t>() + 3,
                                  pool, decode_blocks, st);
      case 12:
        return launch_inflate<12>(ring, ctas_per_sm, job_sync, cur_in, descs.as<ChunkDesc>(), results.as<ChunkResult>(),
                                  work.as<uint32_t>(), d_work_count, counters.as<uint32_t>() + 3,
                                  pool, decode_blocks, st);
      default:
        return launch_inflate<10>(ring, ctas_per_sm, job_sync, cur_in, descs.as<ChunkDesc>(), results.as<ChunkResult>(),
                                  work.as<uint32_t>(), d_work_count, counters.as<uint32_t>() + 3,
                                  pool, decode_blocks, st);
    }
  }

  int setup_decode_grid() {
    int per_sm = 1;
    switch (lut_bits) {
      case 11: per_sm = inflate_blocks_per_sm<11>(ring, ctas_per_sm); break;
      case 12: per_sm = inflate_blocks_per_sm<12>(ring, ctas_per_sm); break;
      default: per_sm = inflate_blocks_per_sm<10>(ring, ctas_per_sm); break;
    }
    if (per_sm < 1) per_sm = 1;
    decode_blocks = per_sm * sms;
    return kOk;
  }

  int run(const std::vector<StreamSpec>& S, std::vector<StreamOut>& R);
  uint32_t pool_cap() const {
    return (uint32_t)std::min<uint64_t>(pages.cap / (kPageEntries * 2),
                                        std::min(owner.cap, seq.cap) / 4);
  }
  // decode again, in a grown page pool, the chunks of [b, e) that ran out of pages
  int regrow(std::vector<ChunkDesc>& hd, std::vector<ChunkResult>& hr, uint32_t b, uint32_t e,
             float& ms_kernel);
  // run() under the autotuner when it is on
  int job(const std::vector<StreamSpec>& S, std::vector<StreamOut>& R);
  int job_tuned(const std::vector<StreamSpec>& S, std::vector<StreamOut>& R);

  // Autotuner: per kind of job (key), the fastest decode parameters found.
  struct TuneCfg {
    uint64_t chunk_bytes;
    int lut_bits, ctas_per_sm;
  };
  std::map<uint32_t, TuneCfg> tune_cache;
  bool tuning = false;     // a trial run: parameters are forced, no cache lookup
  uint32_t last_key = 0;   // key of the last job
  void apply(const TuneCfg& t) {
    chunk_bytes = t.chunk_bytes;
    lut_bits = t.lut_bits;
    ctas_per_sm = t.ctas_per_sm;
    setup_decode_grid();
  }

  // chunk tables of the last job (diagnostics)
  std::vector<ChunkDesc> last_descs;
  std::vector<ChunkResult> last_results;
};

// shortest partition of a high-ratio member (8 KiB of compressed input)
constexpr uint64_t kMinPartitionBits = 8ull << 13;
// shortest piece of a partition cut by the output estimate (4 KiB of input)
constexpr uint64_t kMinPieceBits = 4ull << 13;

static uint64_t pick_chunk_bytes(uint64_t in_len) {
  // several chunks per decoding warp on large inputs, which the
  // longest-first order balances; smaller chunks for small inputs so the
  // warps still fill.  Measured on the 1 GiB mixed stream, whole decode,
  // one box: 48 KiB 43.5 ms, 40 KiB 44.1, 32 KiB 36.4-38.6, 24 KiB 35.3
  // (the decode's tail shrinks faster than the finder and the per-chunk
  // resolve work grow)
  uint64_t c = 24 << 10;
  if (in_len < (4ull << 20)) c = 16 << 10;
  return c;
}

// Internal statuses that reach a caller as public codes: a page pool that
// could not grow (device memory) and a chunk left undecoded are device
// errors; a decode that ran past its stop is invalid deflate data.
static int public_status(int st) {
  switch (st) {
    case kPoolExhausted:
    case kNotDecoded: return GZGPU_DEVICE_ERROR;
    case kOvershoot: return GZGPU_BAD_DEFLATE;
    default: return st;
  }
}

int gzgpu_ctx::job(const std::vector<StreamSpec>& S, std::vector<StreamOut>& R) {
  const int rc = job_tuned(S, R);
  for (StreamOut& r : R) r.status = public_status(r.status);
  return public_status(rc);
}

int gzgpu_ctx::job_tuned(const std::vector<StreamSpec>& S, std::vector<StreamOut>& R) {
  if (!autotune) return run(S, R);
  uint64_t total_in = 0;
  for (const StreamSpec& s : S) total_in += s.len;
  // jobs of a kind not tuned yet start from the defaults
  const TuneCfg dflt{pick_chunk_bytes(total_in), 10, 3};
  apply(dflt);
  int rc = run(S, R);
  if (rc != kOk || tune_cache.count(last_key)) return rc;
  // Coordinate search, one full decode per candidate (outputs are identical,
  // so any run's result stands): chunk size, then LUT bits, then warps/SM.
  const uint32_t key = last_key;
  uint32_t trials = 0;
  auto trial = [&](const TuneCfg& t) {
    apply(t);
    tuning = true;
    auto t0 = std::chrono::steady_clock::now();
    int r = run(S, R);
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    tuning = false;
    trials++;
    return r == kOk ? ms : 1e30;
  };
  TuneCfg best = dflt;
  double best_ms = trial(best);
  for (uint64_t cb : {16ull << 10, 32ull << 10, 64ull << 10, 128ull << 10}) {
    if (cb == best.chunk_bytes) continue;
    TuneCfg t = best;
    t.chunk_bytes = cb;
    double ms = trial(t);
    if (ms < best_ms) best_ms = ms, best = t;
  }
  for (int lb : {11, 12}) {
    TuneCfg t = best;
    t.lut_bits = lb;
    double ms = trial(t);
    if (ms < best_ms) best_ms = ms, best = t;
  }
  {
    TuneCfg t = best;
    t.ctas_per_sm = 4;
    double ms = trial(t);
    if (ms < best_ms) best_ms = ms, best = t;
  }
  tune_cache[key] = best;
  // the final decode with the chosen parameters gives the call's stats
  apply(best);
  stats = gzgpu_stats{};
  rc = run(S, R);
  stats.tune_trials = trials;
  return rc;
}

int gzgpu_ctx::regrow(std::vector<ChunkDesc>& hd, std::vector<ChunkResult>& hr, uint32_t b,
                      uint32_t e, float& ms_kernel) {
  int rc;
  for (;;) {
    std::vector<uint32_t> ids;
    uint64_t extra = 0;  // pages the failed chunks are expected to need
    for (uint32_t i = b; i < e; i++) {
      if (!(hd[i].flags & kChunkValid) || hr[i].status != kPoolExhausted) continue;
      ids.push_back(i);
      const ChunkDesc& d = hd[i];
      const ChunkResult& r = hr[i];
      // output so far, extrapolated over the chunk's compressed range, and
      // never above deflate's ceiling of 1032 output bytes per input byte
      const uint64_t end = std::min<uint64_t>(d.stop_lo, d.in_end * 8);
      const uint64_t span = end > d.start_bit ? end - d.start_bit : 8;
      const uint64_t done = r.end_bit > d.start_bit ? r.end_bit - d.start_bit : 1;
      const double want = (double)r.out_len * (double)span / (double)done * 1.25;
      const double ceil = 1032.0 * (double)span / 8.0 + 258.0;
      extra += (uint64_t)(std::min(want, ceil) / kPageEntries) + 3;
      if ((d.flags >> kGenBaseShift) + 2 * kMaxTries > kGenBaseMax) return kPoolExhausted;
    }
    if (ids.empty()) return kOk;
    uint32_t used = 0;
    if ((rc = check(cudaMemcpyAsync(&used, counters.as<uint32_t>() + 2, 4, cudaMemcpyDeviceToHost,
                                    st))) ||
        (rc = check(cudaStreamSynchronize(st))))
      return rc;
    const uint64_t cap0 = pool_cap();
    used = (uint32_t)std::min<uint64_t>(used, cap0);
    const uint64_t need = std::max<uint64_t>(used + extra + 64, cap0 + cap0 / 4);
    if (need >= kNoPage) return kPoolExhausted;
    if ((rc = check(pages.grow_keep(need * kPageEntries * 2, (uint64_t)used * kPageEntries * 2))) ||
        (rc = check(owner.grow_keep(4 * need, 4ull * used))) ||
        (rc = check(seq.grow_keep(4 * need, 4ull * used))))
      return rc;
    stats.pool_regrows++;
    // the failed chunks start over with attempt numbers past their old pages'
    for (uint32_t i : ids) {
      const uint32_t g = std::min<uint32_t>(hr[i].gen + 1, kGenBaseMax);
      hd[i].flags = (hd[i].flags & ((1u << kGenBaseShift) - 1)) | (g << kGenBaseShift);
      cudaMemcpyAsync(descs.as<ChunkDesc>() + i, &hd[i], sizeof(ChunkDesc), cudaMemcpyHostToDevice, st);
    }
    const uint32_t nw = (uint32_t)ids.size();
    cudaMemcpyAsync(work.p, ids.data(), 4ull * nw, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(counters.as<uint32_t>() + 1, &nw, 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(counters.as<uint32_t>() + 2, &used, 4, cudaMemcpyHostToDevice, st);
    cudaEventRecord(ev[8], st);
    if ((rc = check(launch_decode(counters.as<uint32_t>() + 1)))) return rc;
    cudaEventRecord(ev[9], st);
    cudaMemcpyAsync(hd.data() + b, descs.as<ChunkDesc>() + b, sizeof(ChunkDesc) * (e - b),
                    cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hr.data() + b, results.as<ChunkResult>() + b, sizeof(ChunkResult) * (e - b),
                    cudaMemcpyDeviceToHost, st);
    if ((rc = check(cudaStreamSynchronize(st)))) return rc;
    float t = 0;
    cudaEventElapsedTime(&t, ev[8], ev[9]);
    ms_kernel += t;
  }
}

int gzgpu_ctx::run(const std::vector<StreamSpec>& S, std::vector<StreamOut>& R) {
  const uint32_t ns = (uint32_t)S.size();
  R.assign(ns, StreamOut{});
  int rc;
  auto t_host0 = std::chrono::steady_clock::now();
  cudaEventRecord(ev[1], st);
  // ---- 1. stream headers + member scan --------------------------------
  std::vector<uint64_t> h_off(ns), h_len(ns);
  uint64_t total_in = 0;
  for (uint32_t s = 0; s < ns; s++) {
    h_off[s] = S[s].off;
    h_len[s] = S[s].len;
    total_in += S[s].len;
  }
  std::vector<ScanUnit> units;
  const uint64_t kUnit = 1 << 20;
  for (uint32_t s = 0; s < ns; s++)
    for (uint64_t b = 0; b < S[s].len; b += kUnit)
      units.push_back(ScanUnit{s, 0, b, std::min(S[s].len, b + kUnit)});
  if ((rc = check(s_off.ensure(8 * ns))) || (rc = check(s_len.ensure(8 * ns))) ||
      (rc = check(info.ensure(sizeof(StreamInfo) * ns))) ||
      (rc = check(units.empty() ? cudaSuccess : this->units.ensure(sizeof(ScanUnit) * units.size()))) ||
      (rc = check(counters.ensure(64))))
    return rc;
  uint32_t cand_cap = (uint32_t)std::min<uint64_t>(total_in / 4096 + 4096, 1u << 22);
  if ((rc = check(cands.ensure(sizeof(MemberCand) * cand_cap)))) return rc;
  cudaMemcpyAsync(s_off.p, h_off.data(), 8 * ns, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s_len.p, h_len.data(), 8 * ns, cudaMemcpyHostToDevice, st);
  if (!units.empty())
    cudaMemcpyAsync(this->units.p, units.data(), sizeof(ScanUnit) * units.size(),
                    cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(counters.p, 0, 64, st);
  std::vector<StreamInfo> hinfo(ns);
  uint32_t n_cand = 0;
  if (job_raw) {
    // raw DEFLATE: no header to check and no members to find; each stream
    // is one member whose data starts at its first bit
    for (StreamInfo& h : hinfo) h = StreamInfo{kOk, 0, 0, 4};
  } else {
    if ((rc = check(launch_stream_headers(cur_in, s_off.as<uint64_t>(), s_len.as<uint64_t>(),
                                          ns, info.as<StreamInfo>(), st))))
      return rc;
    if ((rc = check(launch_member_scan(cur_in, this->units.as<ScanUnit>(),
                                       (uint32_t)units.size(), s_off.as<uint64_t>(),
                                       s_len.as<uint64_t>(), info.as<StreamInfo>(),
                                       cands.as<MemberCand>(), counters.as<uint32_t>(), cand_cap,
                                       sms, st))))
      return rc;
    stats.kernel_launches += 2;
    cudaMemcpyAsync(hinfo.data(), info.p, sizeof(StreamInfo) * ns, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&n_cand, counters.p, 4, cudaMemcpyDeviceToHost, st);
  }
  if ((rc = check(cudaStreamSynchronize(st)))) return rc;
  cudaEventRecord(ev[2], st);
  if (autotune) {
    // the kind of job: compressed size (log2), stream count (log4) and the
    // share of streams whose first block is fixed-Huffman (the finder has
    // nothing to find in fixed blocks, so such streams split less)
    uint64_t n_ok = 0, n_fixed = 0;
    for (uint32_t s = 0; s < ns; s++)
      if (hinfo[s].status == kOk) {
        n_ok++;
        n_fixed += hinfo[s].first_btype == 1;
      }
    uint32_t sb = 0, nb = 0;
    while (sb < 63 && (2ull << sb) <= total_in) sb++;
    while (nb < 15 && (4ull << (2 * nb)) <= ns) nb++;
    const uint32_t fb = n_ok ? (uint32_t)((n_fixed * 4 + n_ok / 2) / n_ok) : 0;
    last_key = (sb << 8) | (nb << 4) | fb;
    stats.tune_key = last_key;
    if (!tuning) {
      auto it = tune_cache.find(last_key);
      if (it != tune_cache.end()) apply(it->second);
    }
  }
  n_cand = std::min(n_cand, cand_cap);
  std::vector<MemberCand> hc(n_cand);
  if (n_cand) {
    cudaMemcpyAsync(hc.data(), cands.p, sizeof(MemberCand) * n_cand, cudaMemcpyDeviceToHost, st);
    if ((rc = check(cudaStreamSynchronize(st)))) return rc;
    std::sort(hc.begin(), hc.end(), [](const MemberCand& a, const MemberCand& b) {
      return a.stream != b.stream ? a.stream < b.stream : a.pos < b.pos;
    });
  }
  // ---- 2. members + chunk grid (host) -----------------------------------
  struct Mem {
    uint64_t start, ds, end;
    uint32_t isize;
  };
  std::vector<std::vector<Mem>> mems(ns);
  size_t ci = 0;
  uint64_t est_out = 0;
  for (uint32_t s = 0; s < ns; s++) {
    size_t c_begin = ci;
    while (ci < hc.size() && hc[ci].stream == s) ci++;
    if (hinfo[s].status != kOk) {
      R[s].status = hinfo[s].status == kNotGzip ? kNotGzip : hinfo[s].status;
      continue;
    }
    const uint64_t len = S[s].len;
    std::vector<Mem> ms;
    bool multi = false;
    if (ci - c_begin >= 1 && len >= 18) {
      // scan_member_boundaries_fast acceptance (bgzf.rs:2175-2228)
      multi = true;
      std::vector<uint64_t> starts{0};
      std::vector<uint32_t> hls{hinfo[s].header_len};
      for (size_t k = c_begin; k < ci; k++) {
        starts.push_back(hc[k].pos);
        hls.push_back(hc[k].header_len);
      }
      uint64_t sum_isize = 0;
      for (size_t k = 0; k < starts.size() && multi; k++) {
        uint64_t e = k + 1 < starts.size() ? starts[k + 1] : len;
        if (e - starts[k] < 18 || hls[k] == 0 || starts[k] + hls[k] >= e) {
          multi = false;
          break;
        }
        uint32_t isz = k + 1 < starts.size() ? hc[c_begin + k].prev_isize : hinfo[s].last_isize;
        sum_isize += isz;
        ms.push_back(Mem{starts[k], starts[k] + hls[k], e, isz});
      }
      if (sum_isize > len * 100) multi = false;
    }
    if (!multi) {
      ms.clear();
      ms.push_back(Mem{0, hinfo[s].header_len, len, hinfo[s].last_isize});
    }
    for (auto& m : ms) est_out += m.isize;
    if (job_raw) est_out += 4 * len;  // no ISIZE: the page pool grows if this is short
    mems[s] = std::move(ms);
  }
  // grid
  std::vector<ChunkDesc> hd;
  std::vector<uint32_t> hspec;
  std::vector<uint32_t> c0(ns), c1(ns);
  std::vector<std::vector<uint32_t>> mc0(ns);  // first grid chunk of each planned member
  uint64_t cb = chunk_bytes ? chunk_bytes : pick_chunk_bytes(total_in);
  stats.chunk_bytes = cb;
  stats.lut_bits = lut_bits;
  stats.ctas_per_sm = ring ? 0 : ctas_per_sm;
  const uint64_t cbits = cb * 8;
  for (uint32_t s = 0; s < ns; s++) {
    c0[s] = (uint32_t)hd.size();
    for (const Mem& m : mems[s]) {
      const uint64_t b0 = (S[s].off + m.ds) * 8, bend = (S[s].off + m.end) * 8;
      mc0[s].push_back((uint32_t)hd.size());
      ChunkDesc d{};
      d.start_bit = d.lo_bit = d.guess_bit = b0;
      d.limit_bit = S[s].off + m.start;  // member-first: the member's header byte
      d.stop_lo = kNoStop;
      d.in_end = S[s].off + S[s].len;
      d.flags = kChunkMemberFirst | kChunkValid;
      d.stream = s;
      hd.push_back(d);
      // members that expand a lot (ISIZE over compressed size) get shorter
      // partitions, so chunks carry similar output (about 2 x chunk_bytes)
      uint64_t mbits = cbits;
      const uint64_t clen = m.end > m.ds ? m.end - m.ds : 0;
      if (clen && (uint64_t)m.isize > 2 * clen) {
        mbits = (uint64_t)((double)cbits * 2.0 * (double)clen / (double)m.isize) & ~63ull;
        mbits = std::max<uint64_t>(mbits, std::min<uint64_t>(cbits, kMinPartitionBits));
      }
      for (uint64_t g = b0 + mbits; g < bend; g += mbits) {
        ChunkDesc x{};
        x.start_bit = x.lo_bit = x.guess_bit = g;
        x.limit_bit = std::min(g + mbits, bend);
        x.stop_lo = kNoStop;
        x.in_end = d.in_end;
        x.flags = 0;
        x.stream = s;
        hspec.push_back((uint32_t)hd.size());
        hd.push_back(x);
      }
    }
    c1[s] = (uint32_t)hd.size();
  }
  uint32_t n_grid = (uint32_t)hd.size();
  size_t desc_cap = n_grid + 4096;
  if ((rc = check(descs.ensure(sizeof(ChunkDesc) * desc_cap))) ||
      (rc = check(results.ensure(sizeof(ChunkResult) * desc_cap))) ||
      (rc = check(spec.ensure(4 * (hspec.size() + 1)))) || (rc = check(work.ensure(4 * desc_cap))))
    return rc;
  if (n_grid) cudaMemcpyAsync(descs.p, hd.data(), sizeof(ChunkDesc) * n_grid, cudaMemcpyHostToDevice, st);
  if (!hspec.empty())
    cudaMemcpyAsync(spec.p, hspec.data(), 4 * hspec.size(), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(counters.as<uint32_t>() + 1, 0, 4, st);
  cudaEventRecord(ev[3], st);
  // ---- 3. finder + link ---------------------------------------------------
  uint32_t* n_sync = counters.as<uint32_t>() + 4;  // sync starts found (zeroed with the scan)
  if ((rc = check(launch_finder(cur_in, descs.as<ChunkDesc>(), spec.as<uint32_t>(),
                                (uint32_t)hspec.size(), n_sync, st))))
    return rc;
  stats.kernel_launches += 2;
  // ---- 3a. cut high-ratio partitions finer ---------------------------------
  // A chunk's decode time follows its output; the finder estimated each
  // dynamic start's output per input byte from its code lengths.  Partitions
  // expected to produce more than twice 2 x chunk_bytes are cut into pieces
  // of about that output, which get their own finder pass.
  if (fine_split && !hspec.empty()) {
    if ((rc = check(cudaMemcpyAsync(hd.data(), descs.p, sizeof(ChunkDesc) * n_grid,
                                    cudaMemcpyDeviceToHost, st))) ||
        (rc = check(cudaStreamSynchronize(st))))
      return rc;
    const double target = 2.0 * (double)cb;
    std::vector<ChunkDesc> hd2;
    std::vector<uint32_t> newpos(n_grid + 1), hspec2;
    hd2.reserve(n_grid + n_grid / 4);
    for (uint32_t i = 0; i < n_grid; i++) {
      newpos[i] = (uint32_t)hd2.size();
      hd2.push_back(hd[i]);
      const ChunkDesc& p = hd[i];
      if (!(p.flags & kChunkValid) || (p.flags & (kChunkMemberFirst | kChunkSync)) ||
          !(p.est_ratio > 0.f) || p.limit_bit <= p.start_bit)
        continue;
      // the first block may not represent the partition (a content change
      // inside it): the next partition's first block shows its far end
      float ratio = p.est_ratio;
      if (i + 1 < n_grid && hd[i + 1].stream == p.stream && (hd[i + 1].flags & kChunkValid) &&
          !(hd[i + 1].flags & kChunkMemberFirst))
        ratio = std::max(ratio, hd[i + 1].est_ratio);
      const uint64_t span = p.limit_bit - p.start_bit;
      const double est = (double)ratio * (double)span / 8.0;
      if (est <= 2.0 * target) continue;
      const uint64_t k = std::min<uint64_t>(8, (uint64_t)(est / target + 0.999));
      const uint64_t piece = std::max<uint64_t>((span / k) & ~63ull, kMinPieceBits);
      for (uint64_t g = p.start_bit + piece; g + kMinPieceBits <= p.limit_bit; g += piece) {
        ChunkDesc x{};
        x.start_bit = x.lo_bit = x.guess_bit = g;
        x.limit_bit = std::min(g + piece, p.limit_bit);
        if (p.limit_bit - x.limit_bit < kMinPieceBits) x.limit_bit = p.limit_bit;
        x.stop_lo = kNoStop;
        x.in_end = p.in_end;
        x.stream = p.stream;
        x.flags = kChunkPiece;
        hspec2.push_back((uint32_t)hd2.size());
        hd2.push_back(x);
        if (x.limit_bit == p.limit_bit) break;
      }
    }
    newpos[n_grid] = (uint32_t)hd2.size();
    if (!hspec2.empty()) {
      for (uint32_t s = 0; s < ns; s++) {
        c0[s] = newpos[c0[s]];
        c1[s] = newpos[c1[s]];
        for (uint32_t& m : mc0[s]) m = newpos[m];
      }
      hd.swap(hd2);
      n_grid = (uint32_t)hd.size();
      desc_cap = n_grid + 4096;
      if ((rc = check(descs.ensure(sizeof(ChunkDesc) * desc_cap))) ||
          (rc = check(results.ensure(sizeof(ChunkResult) * desc_cap))) ||
          (rc = check(spec.ensure(4 * (hspec2.size() + 1)))) ||
          (rc = check(work.ensure(4 * desc_cap))))
        return rc;
      cudaMemcpyAsync(descs.p, hd.data(), sizeof(ChunkDesc) * n_grid, cudaMemcpyHostToDevice, st);
      cudaMemcpyAsync(spec.p, hspec2.data(), 4 * hspec2.size(), cudaMemcpyHostToDevice, st);
      if ((rc = check(launch_finder(cur_in, descs.as<ChunkDesc>(), spec.as<uint32_t>(),
                                    (uint32_t)hspec2.size(), n_sync, st))))
        return rc;
      stats.kernel_launches += 2;
    }
    // sync starts inside dynamic blocks for every partition still empty
    std::vector<uint32_t> hsync;
    hsync.reserve(n_grid);
    for (uint32_t i = 0; i < n_grid; i++)
      if (!(hd[i].flags & kChunkMemberFirst)) hsync.push_back(i);
    if (!hsync.empty()) {
      if ((rc = check(spec.ensure(4 * (hsync.size() + 1))))) return rc;
      cudaMemcpyAsync(spec.p, hsync.data(), 4 * hsync.size(), cudaMemcpyHostToDevice, st);
      if ((rc = check(launch_dyn_sync(cur_in, descs.as<ChunkDesc>(), spec.as<uint32_t>(),
                                      (uint32_t)hsync.size(), n_sync, st))))
        return rc;
      stats.kernel_launches += 1;
    }
  }
  stats.n_chunks = n_grid;
  if (lpt && (rc = check(cost.ensure(4 * (size_t)(n_grid + 1))))) return rc;
  if ((rc = check(launch_link(cur_in, descs.as<ChunkDesc>(), n_grid, work.as<uint32_t>(),
                              counters.as<uint32_t>() + 1, lpt ? cost.as<float>() : nullptr,
                              std::max<uint64_t>(cbits, 1ull << 21), st))))
    return rc;
  stats.kernel_launches += lpt ? 2 : 1;
  {
    // the decoder variant without sync-start handling when there are none
    uint32_t h_sync = 1;
    if ((rc = check(cudaMemcpyAsync(&h_sync, n_sync, 4, cudaMemcpyDeviceToHost, st))) ||
        (rc = check(cudaStreamSynchronize(st))))
      return rc;
    job_sync = h_sync != 0;
  }
  cudaEventRecord(ev[4], st);
  // ---- 4. decode ----------------------------------------------------------
  // The pool is sized from the members' ISIZEs (raw streams: 4 x their
  // input).  ISIZE is only a hint (it wraps past 4 GiB, and a raw stream has
  // none): the chunks that run out of pages are decoded again in a grown
  // pool, the others keep theirs (regrow).
  uint64_t pages_needed = (est_out + n_grid * (uint64_t)kPageEntries) / kPageEntries + 64;
  std::vector<ChunkResult> hr;
  float ms_dec_kernel = 0;
  {
    if ((rc = check(pages.ensure(pages_needed * kPageEntries * 2))) ||
        (rc = check(owner.ensure(4 * pages_needed))) || (rc = check(seq.ensure(4 * pages_needed))))
      return rc;
    cudaMemsetAsync(counters.as<uint32_t>() + 2, 0, 4, st);
    if (job_index) {
      blk_cap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(blk_need, total_in / 64 + 65536),
                                             1u << 30);
      if ((rc = check(blk_log.ensure(sizeof(BlockRec) * (uint64_t)blk_cap)))) return rc;
      cudaMemsetAsync(counters.as<uint32_t>() + 8, 0, 4, st);
    }
    cudaEventRecord(ev[8], st);
    if ((rc = check(launch_decode(counters.as<uint32_t>() + 1)))) return rc;
    cudaEventRecord(ev[9], st);
    hd.resize(n_grid);
    hr.resize(n_grid);
    if (n_grid) {
      cudaMemcpyAsync(hd.data(), descs.p, sizeof(ChunkDesc) * n_grid, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(hr.data(), results.p, sizeof(ChunkResult) * n_grid, cudaMemcpyDeviceToHost, st);
    }
    if ((rc = check(cudaStreamSynchronize(st)))) return rc;
    float t = 0;
    cudaEventElapsedTime(&t, ev[8], ev[9]);
    ms_dec_kernel += t;
    if ((rc = regrow(hd, hr, 0, n_grid, ms_dec_kernel))) return rc;
  }
  cudaEventRecord(ev[5], st);
  // ---- 5. chain walk with repairs (host) ---------------------------------
  std::vector<std::vector<Walker>> SW(ns);
  auto whole_stream = [&](uint32_t s) {
    Walker w;
    w.stream = s;
    w.c0 = w.j = c0[s];
    w.c1 = c1[s];
    w.mpos = 0;
    if (R[s].status != kOk || c0[s] == c1[s]) w.done = true;
    return w;
  };
  for (uint32_t s = 0; s < ns; s++) {
    const size_t nm = mc0[s].size();
    if (nm <= 1 || R[s].status != kOk) {
      SW[s].push_back(whole_stream(s));
      continue;
    }
    for (size_t k = 0; k < nm; k++) {
      Walker w;
      w.stream = s;
      w.c0 = w.j = mc0[s][k];
      w.c1 = k + 1 < nm ? mc0[s][k + 1] : c1[s];
      w.mpos = mems[s][k].start;
      w.member = (uint32_t)k;
      w.last = k + 1 == nm;
      w.mend = w.last ? S[s].len : mems[s][k + 1].start;
      SW[s].push_back(w);
    }
  }
  auto is_valid = [&](uint32_t i) { return (hd[i].flags & kChunkValid) != 0; };
  auto is_mf = [&](uint32_t i) { return (hd[i].flags & kChunkMemberFirst) != 0; };
  auto is_sync = [&](uint32_t i) { return (hd[i].flags & kChunkSync) != 0; };
  std::vector<ChunkDesc> repairs;
  std::vector<uint32_t> repair_owner;
  uint64_t n_rejected = 0, n_repairs = 0;
  // bytes of an input range, fetched on demand (rare: members the scan missed)
  auto fetch = [&](uint64_t abs, size_t n, uint8_t* dst) {
    cudaMemcpy(dst, cur_in + abs, n, cudaMemcpyDeviceToHost);
  };
  // a repair starts at a confirmed boundary and stops at the start of grid
  // chunk `next` (kNoChunk: none); like a member-first chunk it decodes on
  // through any phantom successors it finds there
  auto new_chunk = [&](Walker& w, uint64_t start, uint64_t stop, uint32_t flags, uint32_t next,
                       uint64_t table_bit = 0) {
    ChunkDesc d{};
    d.start_bit = d.lo_bit = d.guess_bit = d.limit_bit = start;
    if (flags & kChunkMemberFirst) d.limit_bit = S[w.stream].off + w.mpos;
    d.stop_lo = stop;
    d.abort_bit = kNoStop;
    d.in_end = S[w.stream].off + S[w.stream].len;
    d.flags = flags | kChunkValid | kChunkConfirmed;
    d.stream = w.stream;
    d.next = next;
    d.table_bit = table_bit;
    uint32_t id = (uint32_t)(hd.size() + repairs.size());
    repairs.push_back(d);
    repair_owner.push_back(w.stream);
    w.pending = (int32_t)id;
    n_repairs++;
  };
  // advance one walker as far as possible; returns when done or a repair is pending
  auto step = [&](Walker& w) {
    const uint64_t base = S[w.stream].off, len = S[w.stream].len;
    while (!w.done && w.pending < 0) {
      if (w.cur < 0) {
        // at a member header
        if (w.member > 0 && w.mpos >= len) {
          w.done = true;
          break;
        }
        uint32_t j = w.j;
        while (j < w.c1 && !(is_valid(j) && is_mf(j) && hd[j].limit_bit >= base + w.mpos)) j++;
        bool found = false;
        if (j < w.c1 && hd[j].limit_bit == base + w.mpos) {
          w.cur = (int32_t)j;
          w.j = j + 1;
          found = true;
        }
        if (!found) {
          if (w.member == 0) {
            w.status = kBadHeader;
            w.done = true;
            break;
          }
          uint8_t hb[64] = {0};
          size_t nb = (size_t)std::min<uint64_t>(64, len - w.mpos);
          if (len - w.mpos < 18) {
            w.done = true;  // too short to be a member: stop cleanly
            break;
          }
          fetch(base + w.mpos, nb, hb);
          if (hb[0] != 0x1f || hb[1] != 0x8b || hb[2] != 8 || (hb[3] & 0xE0)) {
            w.done = true;  // trailing bytes that start no member
            break;
          }
          // header length (FEXTRA/FNAME/FCOMMENT may exceed 64 bytes: fetch more)
          uint64_t o = 10;
          uint8_t flg = hb[3];
          std::vector<uint8_t> hbuf;
          size_t want = (size_t)std::min<uint64_t>(len - w.mpos, 1 << 20);
          hbuf.resize(want);
          fetch(base + w.mpos, want, hbuf.data());
          bool ok = true;
          if (flg & 4) {
            if (o + 2 > want) ok = false;
            else o += 2 + (hbuf[o] | (hbuf[o + 1] << 8));
          }
          for (int f = 8; f <= 16 && ok; f <<= 1)
            if (flg & f) {
              while (o < want && hbuf[o]) o++;
              if (o >= want) ok = false;
              o++;
            }
          if (ok && (flg & 2)) o += 2;
          if (!ok || o >= want) {
            w.done = true;
            break;
          }
          w.member_order_begin = (uint32_t)w.order.size();
          new_chunk(w, (base + w.mpos + o) * 8, kNoStop, kChunkMemberFirst, kNoChunk);
          break;
        }
        w.member_order_begin = (uint32_t)w.order.size();
      }
      // inside a member
      const uint32_t cur = (uint32_t)w.cur;
      const ChunkResult& r = hr[cur];
      w.order.push_back(cur);
      if (r.status != kOk) {
        w.status = r.status;
        w.done = true;
        break;
      }
      if (r.final_block && job_raw) {
        // raw DEFLATE ends with its final block; bytes after it are ignored
        if ((r.end_bit + 7) / 8 > base + len) w.status = kTruncated;
        else w.members.push_back(MemberPlan{w.member_order_begin, (uint32_t)w.order.size(), kNoTrailer, 0});
        w.done = true;
        break;
      }
      if (r.final_block) {
        uint64_t trailer = (r.end_bit + 7) / 8;
        if (trailer + 8 > base + len) {
          w.status = kTruncated;
          w.done = true;
          break;
        }
        w.members.push_back(MemberPlan{w.member_order_begin, (uint32_t)w.order.size(), trailer, 0});
        w.member++;
        w.mpos = trailer + 8 - base;
        w.cur = -1;
        if (!w.last) {
          // a segment hands over exactly at the next planned member
          w.handoff_bad = w.mpos != w.mend;
          w.done = true;
          break;
        }
        continue;
      }
      // accept the chunk whose start range holds the confirmed end; discard
      // the starts the end passed (phantom speculative starts, and member
      // candidates that lay inside this member's data)
      const uint64_t e = r.end_bit;
      auto first_bit = [&](uint32_t k) { return is_mf(k) ? hd[k].limit_bit * 8 : hd[k].lo_bit; };
      uint32_t j = w.j;
      bool accepted = false;
      while (j < w.c1) {
        if (!is_valid(j)) {
          j++;
          continue;
        }
        // a sync start is taken over only by a chunk that stopped at it
        // mid-block, any other start only at a block boundary
        if (!is_mf(j) && e >= hd[j].lo_bit && e <= hd[j].start_bit && hr[j].status == kOk &&
            is_sync(j) == (r.sync_end != 0)) {
          accepted = true;
          break;
        }
        if (first_bit(j) > e) break;
        n_rejected++;
        j++;
      }
      if (accepted) {
        w.cur = (int32_t)j;
        w.j = j + 1;
        continue;
      }
      w.j = j;
      uint64_t stop = j < w.c1 ? first_bit(j) : kNoStop;
      if (j < w.c1 && !is_mf(j) && hr[j].status == kOk) {
        // optimistic: the repair ends at the next candidate's start
        Walker::Checkpoint cp{w.order.size(), w.members.size(), j, w.member,
                              w.member_order_begin, w.mpos};
        new_chunk(w, e, stop, r.sync_end ? kChunkSync : 0u, j, r.sync_end ? r.end_hdr_bit : 0);
        uint32_t rid = (uint32_t)w.pending;
        w.pending = -1;
        w.assumed.push_back(Walker::Assumption{rid, hd[j].lo_bit, hd[j].start_bit, is_sync(j), cp});
        w.order.push_back(rid);
        w.cur = (int32_t)j;
        w.j = j + 1;
        continue;
      }
      new_chunk(w, e, stop, r.sync_end ? kChunkSync : 0u, j < w.c1 ? j : kNoChunk,
                r.sync_end ? r.end_hdr_bit : 0);
      break;
    }
  };
  for (;;) {
    for (auto& sw : SW)
      for (auto& w : sw) step(w);
    // a segment that ended off its planned hand-over (or failed in a way
    // that leaves it unverified) sends its stream back to one whole walk
    bool rewalk = false;
    for (uint32_t s = 0; s < ns; s++) {
      bool bad = false;
      for (auto& w : SW[s])  // decided once its optimistic repairs are verified
        bad |= w.handoff_bad && (w.assumed.empty() || w.assumed.back().repair < hd.size());
      if (bad) {
        SW[s].clear();
        SW[s].push_back(whole_stream(s));
        rewalk = true;
      }
    }
    if (rewalk) continue;
    if (repairs.empty()) break;
    // decode all pending repairs in one pass
    const uint32_t base_id = (uint32_t)hd.size(), nr = (uint32_t)repairs.size();
    if (hd.size() + nr > desc_cap) {
      // grow device arrays, preserving contents
      size_t ncap = (hd.size() + nr) * 2;
      DevBuf nd, nrr;
      nd.st = nrr.st = st;
      if ((rc = check(nd.ensure(sizeof(ChunkDesc) * ncap))) ||
          (rc = check(nrr.ensure(sizeof(ChunkResult) * ncap))))
        return rc;
      cudaMemcpyAsync(nd.p, descs.p, sizeof(ChunkDesc) * hd.size(), cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(nrr.p, results.p, sizeof(ChunkResult) * hd.size(), cudaMemcpyDeviceToDevice, st);
      cudaStreamSynchronize(st);
      descs.release();
      results.release();
      descs = nd;
      results = nrr;
      if ((rc = check(work.ensure(4 * ncap)))) return rc;
      desc_cap = ncap;
    }
    std::vector<uint32_t> wl(nr);
    for (uint32_t k = 0; k < nr; k++) wl[k] = base_id + k;
    cudaMemcpyAsync(descs.as<ChunkDesc>() + base_id, repairs.data(), sizeof(ChunkDesc) * nr,
                    cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(work.p, wl.data(), 4 * nr, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(counters.as<uint32_t>() + 1, &nr, 4, cudaMemcpyHostToDevice, st);
    cudaEventRecord(ev[8], st);
    if ((rc = check(launch_decode(counters.as<uint32_t>() + 1)))) return rc;
    cudaEventRecord(ev[9], st);
    hd.insert(hd.end(), repairs.begin(), repairs.end());
    hr.resize(hd.size());
    cudaMemcpyAsync(hr.data() + base_id, results.as<ChunkResult>() + base_id,
                    sizeof(ChunkResult) * nr, cudaMemcpyDeviceToHost, st);
    if ((rc = check(cudaStreamSynchronize(st)))) return rc;
    float t = 0;
    cudaEventElapsedTime(&t, ev[8], ev[9]);
    ms_dec_kernel += t;
    if ((rc = regrow(hd, hr, base_id, base_id + nr, ms_dec_kernel))) return rc;
    for (auto& sw : SW) {
      for (Walker& w : sw) {
        if (w.pending >= 0) {
          w.cur = w.pending;
          w.pending = -1;
        }
        for (size_t a = 0; a < w.assumed.size(); a++) {
          const Walker::Assumption& as = w.assumed[a];
          if (as.repair < base_id) continue;  // verified in an earlier pass
          const ChunkResult& rr = hr[as.repair];
          if (rr.status == kOk && !rr.final_block && rr.end_bit >= as.lo && rr.end_bit <= as.hi &&
              (rr.sync_end != 0) == as.sync)
            continue;
          // the repair ended elsewhere: resume the walk from it
          w.order.resize(as.cp.order_size);
          w.members.resize(as.cp.members_size);
          w.j = as.cp.j;
          w.member = as.cp.member;
          w.member_order_begin = as.cp.member_order_begin;
          w.mpos = as.cp.mpos;
          w.cur = (int32_t)as.repair;
          w.done = false;
          w.handoff_bad = false;
          w.status = kOk;
          w.assumed.resize(a);
          break;
        }
      }
    }
    repairs.clear();
    repair_owner.clear();
  }
  stats.n_rejected = n_rejected;
  stats.n_repairs = n_repairs;
  last_descs = hd;
  last_results = hr;
  // ---- output placement ----------------------------------------------------
  const uint32_t n_all = (uint32_t)hd.size();
  std::vector<PlacedChunk> placed;
  std::vector<uint32_t> placed_of(n_all, 0xFFFFFFFFu);
  std::vector<uint32_t> tlist;  // placed chunks whose tails hold markers
  std::vector<CrcBlock> cblk;
  std::vector<uint64_t> mtrail, mlenv, mendv;
  uint64_t out_total = 0;
  for (uint32_t s = 0; s < ns; s++) {
    for (Walker& w : SW[s])
      if (R[s].status == kOk) R[s].status = w.status;
    if (R[s].status != kOk) continue;
    R[s].out_off = out_total;
    uint64_t so = 0;
    for (Walker& w : SW[s]) for (MemberPlan& mp : w.members) {
      mp.out_len = 0;
      for (uint32_t k = mp.order_begin; k < mp.order_end; k++) mp.out_len += hr[w.order[k]].out_len;
      uint64_t moff = out_total + so;
      for (uint32_t k = mp.order_begin; k < mp.order_end; k++) {
        uint32_t cid = w.order[k];
        placed_of[cid] = (uint32_t)placed.size();
        placed.push_back(PlacedChunk{out_total + so, moff, cid, 0});
        const ChunkResult& r = hr[cid];
        uint64_t t0 = r.out_len > kWindow ? r.out_len - kWindow : 0;
        if (r.marker_end > t0) tlist.push_back((uint32_t)placed.size() - 1);
        so += r.out_len;
      }
      for (uint64_t b = 0; mp.trailer != kNoTrailer && b < mp.out_len; b += kCrcBlock)
        cblk.push_back(CrcBlock{moff + b, (uint32_t)std::min<uint64_t>(kCrcBlock, mp.out_len - b),
                                (uint32_t)mtrail.size()});
      mtrail.push_back(mp.trailer);
      mlenv.push_back(mp.out_len);
      mendv.push_back(moff + mp.out_len);
    }
    R[s].out_len = so;
    out_total += so;
  }
  stats.n_accepted = placed.size();
  stats.n_tail_marker_chunks = tlist.size();
  stats.n_members = mtrail.size();
  stats.out_bytes = out_total;
  cudaEventRecord(ev[6], st);
  // ---- 6. resolve + CRC ----------------------------------------------------
  uint32_t n_pages_used = 0;
  cudaMemcpyAsync(&n_pages_used, counters.as<uint32_t>() + 2, 4, cudaMemcpyDeviceToHost, st);
  if ((rc = check(cudaStreamSynchronize(st)))) return rc;
  const uint32_t pcap = pool_cap();
  n_pages_used = std::min(n_pages_used, pcap);
  stats.n_pages = n_pages_used;
  cur_out = (user_out && out_total <= user_cap) ? user_out : nullptr;
  if ((rc = check(cur_out ? cudaSuccess : out.ensure(out_total + 64))) ||
      (rc = check(this->placed.ensure(sizeof(PlacedChunk) * (placed.size() + 1)))) ||
      (rc = check(this->placed_of.ensure(4 * (n_all + 1)))) || (rc = check(list.ensure(4 * (tlist.size() + 1)))) ||
      (rc = check(cblocks.ensure(sizeof(CrcBlock) * (cblk.size() + 1)))) ||
      (rc = check(mend.ensure(8 * (mendv.size() + 1)))) || (rc = check(mraw.ensure(4 * (mtrail.size() + 1)))) ||
      (rc = check(this->mtrail.ensure(8 * (mtrail.size() + 1)))) || (rc = check(mlen.ensure(8 * (mlenv.size() + 1)))) ||
      (rc = check(mcrc.ensure(4 * (mtrail.size() + 1)))) ||
      (rc = check(mstatus.ensure(4 * (mtrail.size() + 1)))))
    return rc;
  if (!placed.empty())
    cudaMemcpyAsync(this->placed.p, placed.data(), sizeof(PlacedChunk) * placed.size(),
                    cudaMemcpyHostToDevice, st);
  if (n_all) cudaMemcpyAsync(this->placed_of.p, placed_of.data(), 4 * n_all, cudaMemcpyHostToDevice, st);
  if (!tlist.empty()) cudaMemcpyAsync(list.p, tlist.data(), 4 * tlist.size(), cudaMemcpyHostToDevice, st);
  if (!cblk.empty())
    cudaMemcpyAsync(cblocks.p, cblk.data(), sizeof(CrcBlock) * cblk.size(), cudaMemcpyHostToDevice, st);
  if (!mtrail.empty()) {
    cudaMemcpyAsync(this->mtrail.p, mtrail.data(), 8 * mtrail.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(mlen.p, mlenv.data(), 8 * mlenv.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(mend.p, mendv.data(), 8 * mendv.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(mraw.p, 0, 4 * mtrail.size(), st);
  }
  if (!cur_out) cur_out = out.as<uint8_t>();
  PagePool pool{pages.as<uint16_t>(), owner.as<uint32_t>(), seq.as<uint32_t>(),
                counters.as<uint32_t>() + 2, pcap};
  cudaEventRecord(ev[10], st);
  if (!crc_ready) {
    if ((rc = check(resolve_init(st)))) return rc;
    crc_ready = true;
  }
  const uint32_t np = (uint32_t)placed.size();
  if ((rc = check(launch_tail_literals(this->placed.as<PlacedChunk>(), np, results.as<ChunkResult>(),
                                       pool, cur_out, st))) ||
      (rc = check(launch_tail_markers(this->placed.as<PlacedChunk>(), list.as<uint32_t>(),
                                      (uint32_t)tlist.size(), results.as<ChunkResult>(), pool,
                                      cur_out, sms, st))) ||
      (rc = check(launch_body(this->placed.as<PlacedChunk>(), this->placed_of.as<uint32_t>(),
                              n_pages_used, results.as<ChunkResult>(), pool, cur_out, sms,
                              st))))
    return rc;
  cudaEventRecord(ev[11], st);
  if ((rc = check(launch_crc(cblocks.as<CrcBlock>(), (uint32_t)cblk.size(), cur_out,
                             mend.as<uint64_t>(), mraw.as<uint32_t>(),
                             this->mtrail.as<uint64_t>(), mlen.as<uint64_t>(),
                             (uint32_t)mtrail.size(), cur_in, mcrc.as<uint32_t>(),
                             mstatus.as<int32_t>(), sms, st))))
    return rc;
  stats.kernel_launches += 5;
  std::vector<int32_t> mst(mtrail.size());
  if (!mst.empty())
    cudaMemcpyAsync(mst.data(), mstatus.p, 4 * mst.size(), cudaMemcpyDeviceToHost, st);
  cudaEventRecord(ev[7], st);
  if ((rc = check(cudaStreamSynchronize(st)))) return rc;
  {
    size_t mi = 0;
    for (uint32_t s = 0; s < ns; s++) {
      if (R[s].status != kOk) continue;
      size_t nm = 0;
      for (const Walker& w : SW[s]) nm += w.members.size();
      for (size_t k = 0; k < nm; k++, mi++)
        if (R[s].status == kOk && mst[mi] != kOk) R[s].status = mst[mi];
    }
  }
  if (job_index) {
    // seek index (build_index / scan_deflate, src/decompress/index.rs:55-141,
    // src/decompress/scan_inflate.rs:46-130): walk the blocks of the one
    // member in output order; at a block start whose output offset has
    // reached the next checkpoint (and at least one window), record the
    // header's bit (from the deflate start), the offset and the 32 KiB of
    // output before it
    index_bytes.clear();
    index_status = kOk;
    size_t n_mem = 0;
    if (ns == 1)
      for (const Walker& w : SW[0]) n_mem += w.members.size();
    if (ns != 1 || R[0].status != kOk || n_mem != 1) {
      index_status = ns == 1 && R[0].status != kOk ? R[0].status : GZGPU_INVALID_ARGUMENT;
    } else {
      uint32_t nrec = 0;
      if ((rc = check(cudaMemcpyAsync(&nrec, counters.as<uint32_t>() + 8, 4, cudaMemcpyDeviceToHost, st))) ||
          (rc = check(cudaStreamSynchronize(st))))
        return rc;
      if (nrec > blk_cap) {
        blk_need = nrec + nrec / 4 + 1024;  // the caller decodes again with a larger log
        index_status = kPoolExhausted;
      } else {
        std::vector<BlockRec> recs(nrec);
        if (nrec && ((rc = check(cudaMemcpyAsync(recs.data(), blk_log.p, sizeof(BlockRec) * nrec,
                                                 cudaMemcpyDeviceToHost, st))) ||
                     (rc = check(cudaStreamSynchronize(st)))))
          return rc;
        std::sort(recs.begin(), recs.end(), [](const BlockRec& a, const BlockRec& b) {
          return a.chunk != b.chunk ? a.chunk < b.chunk : a.hdr_bit < b.hdr_bit;
        });
        const uint64_t deflate_bit = (S[0].off + hinfo[0].header_len) * 8;
        const uint64_t interval = index_interval;
        uint64_t next_cp = interval;
        std::vector<std::pair<uint64_t, uint64_t>> pts;  // (bit from the deflate start, output offset)
        uint64_t prev_end = kNoStop;
        for (const PlacedChunk& p : placed) {
          const uint32_t cid = p.chunk;
          auto it = std::lower_bound(recs.begin(), recs.end(), cid,
                                     [](const BlockRec& a, uint32_t c) { return a.chunk < c; });
          uint64_t last_bit = kNoStop;
          for (; it != recs.end() && it->chunk == cid; ++it) {
            // the accepted attempt's blocks inside its decoded range, once each
            if (it->gen != hr[cid].gen || it->hdr_bit < hd[cid].start_bit || it->hdr_bit >= hr[cid].end_bit ||
                it->hdr_bit == last_bit)
              continue;
            last_bit = it->hdr_bit;
            // a chunk accepted from a start range (a stored block's header
            // and padding bits) began where its predecessor ended: that bit
            // is the block's boundary in the stream
            uint64_t bit = it->hdr_bit;
            if (bit == hd[cid].start_bit && !(hd[cid].flags & kChunkMemberFirst) && prev_end != kNoStop)
              bit = prev_end;
            const uint64_t out = p.out_off - R[0].out_off + it->out_pos;
            if (out >= next_cp && out >= kWindow) {
              pts.emplace_back(bit - deflate_bit, out);
              next_cp = out + interval;
            }
          }
          prev_end = hr[cid].end_bit;
        }
        const bool none = pts.empty();
        if (none) pts.emplace_back(0, 0);  // one point at the start (index.rs:124-134)
        constexpr size_t kPoint = 8 + 8 + kWindow;
        index_bytes.assign(6 + 4 + 8 + 4 + 2 + pts.size() * kPoint, 0);
        uint8_t* q = index_bytes.data();
        auto put = [&](uint64_t v, int n) {
          for (int i = 0; i < n; i++) *q++ = (uint8_t)(v >> (8 * i));
        };
        memcpy(q, "GZIDX\x01", 6);
        q += 6;
        put(hinfo[0].header_len, 4);
        put(R[0].out_len, 8);
        put(pts.size(), 4);
        put(0, 2);
        for (const auto& pt : pts) {
          put(pt.first, 8);
          put(pt.second, 8);
          if (!none &&
              (rc = check(cudaMemcpyAsync(q, cur_out + R[0].out_off + pt.second - kWindow, kWindow,
                                          cudaMemcpyDeviceToHost, st))))
            return rc;
          q += kWindow;
        }
        if ((rc = check(cudaStreamSynchronize(st)))) return rc;
      }
    }
  }
  float t;
  auto el = [&](int a, int b) {
    t = 0;
    cudaEventElapsedTime(&t, ev[a], ev[b]);
    return (double)t;
  };
  stats.ms_scan = el(1, 2);
  stats.ms_find = el(3, 4);
  stats.ms_decode = el(4, 5);
  stats.ms_decode_kernel = ms_dec_kernel;
  stats.ms_walk = el(5, 6);
  stats.ms_resolve = el(10, 11);
  stats.ms_crc = el(11, 7);
  stats.n_streams = ns;
  stats.in_bytes = total_in;
  (void)t_host0;
  return kOk;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* gzgpu_strerror(int code) {
  if (code >= 0 && code < (int)(sizeof(kErrStr) / sizeof(kErrStr[0]))) return kErrStr[code];
  return "unknown error";
}

int gzgpu_create(gzgpu_ctx** out, const gzgpu_config* cfg) {
  if (!out) return GZGPU_INVALID_ARGUMENT;
  *out = nullptr;
  gzgpu_ctx* c = new (std::nothrow) gzgpu_ctx();
  if (!c) return GZGPU_DEVICE_ERROR;
  if (cfg) {
    c->dev = cfg->device;
    c->chunk_bytes = cfg->chunk_bytes;
    if (cfg->lut_bits == 11 || cfg->lut_bits == 12) c->lut_bits = cfg->lut_bits;
    c->autotune = cfg->autotune != 0;
    c->ring = cfg->ring_history != 0;
    if (cfg->ctas_per_sm == 3 || cfg->ctas_per_sm == 4) c->ctas_per_sm = cfg->ctas_per_sm;
    c->fine_split = cfg->fine_split != 0;
    c->high_priority = cfg->high_priority != 0;
    c->lpt = cfg->work_order == 0;
    // decoder 1: lane-parallel 32-bit steps, 2: serial, 3: 64-bit steps,
    // 4: chosen per block
    static const uint32_t kMode[5] = {0u, 0u, 1u, 2u, 3u};
    if (cfg->decoder >= 1 && cfg->decoder <= 4) c->decoder_mode = kMode[cfg->decoder];
  }
  if (cudaSetDevice(c->dev) != cudaSuccess) {
    delete c;
    return GZGPU_DEVICE_ERROR;
  }
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev);
  int prio_least = 0, prio_greatest = 0;
  cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (cudaStreamCreateWithPriority(&c->st, cudaStreamNonBlocking,
                                   c->high_priority ? prio_greatest : prio_least) != cudaSuccess) {
    delete c;
    return GZGPU_DEVICE_ERROR;
  }
  for (auto& e : c->ev) cudaEventCreate(&e);
  for (auto& e : c->stage_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (DevBuf* b : c->all_bufs()) b->st = c->st;
  {
    // keep memory freed by buffer growth in the device's pool for reuse
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, c->dev) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  c->setup_decode_grid();
  *out = c;
  return GZGPU_OK;
}

void gzgpu_destroy(gzgpu_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->st);
  for (DevBuf* b : c->all_bufs()) b->release();
  cudaStreamSynchronize(c->st);
  c->h_stage.release();
  for (auto& e : c->ev) cudaEventDestroy(e);
  for (auto& e : c->stage_ev) cudaEventDestroy(e);
  cudaStreamDestroy(c->st);
  delete c;
}

namespace {

void reset_stats(gzgpu_ctx* c) {
  c->stats = gzgpu_stats{};
  c->stats.lut_bits = c->lut_bits;
}

void finish_stats(gzgpu_ctx* c) {
  float t = 0;
  cudaEventElapsedTime(&t, c->ev[0], c->ev[1]);
  c->stats.ms_h2d = t;
  t = 0;
  cudaEventElapsedTime(&t, c->ev[0], c->ev[7]);
  c->stats.ms_total = t;
}

}  // namespace

namespace {

// Host copies: a stream in page-locked memory (in the batch path, one of at
// least kDirectBytes) moves by DMA straight from / to the caller's buffer;
// the others go through the context's pinned staging ring (stage.h: two
// kStageSlot slots, allocated once), gathered and scattered by up to
// kCopyThreads host threads while the other slot's DMA runs.
constexpr size_t kDirectBytes = 1u << 20;
constexpr int kCopyThreads = 16;

bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // pageable memory of an old driver reports an error: clear it
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

struct CopyJob {
  void* dst;
  const void* src;
  size_t len;
};

void parallel_copy(const std::vector<CopyJob>& jobs) {
  size_t total = 0;
  for (const CopyJob& j : jobs) total += j.len;
  int nt = (int)std::min<size_t>(kCopyThreads, total / (2u << 20) + 1);
  nt = std::max(1, std::min(nt, (int)std::thread::hardware_concurrency()));
  if (nt <= 1) {
    for (const CopyJob& j : jobs) memcpy(j.dst, j.src, j.len);
    return;
  }
  // split the byte range evenly; a job may be cut between threads
  const size_t per = (total + nt - 1) / nt;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; t++) {
    th.emplace_back([&, t] {
      const size_t b0 = t * per, b1 = std::min(total, b0 + per);
      size_t at = 0;
      for (const CopyJob& j : jobs) {
        const size_t j0 = at, j1 = at + j.len;
        at = j1;
        if (j1 <= b0 || j0 >= b1) continue;
        const size_t s0 = std::max(j0, b0) - j0, s1 = std::min(j1, b1) - j0;
        memcpy((uint8_t*)j.dst + s0, (const uint8_t*)j.src + s0, s1 - s0);
      }
    });
  }
  for (std::thread& x : th) x.join();
}

// the staging ring's device side: copies and slot events on the context stream
struct CudaStageOps {
  gzgpu_ctx* c;
  uint8_t* dev;  // device base of the staged byte offsets
  int to_dev(uint64_t d, const uint8_t* src, uint64_t len) {
    return c->check(cudaMemcpyAsync(dev + d, src, len, cudaMemcpyHostToDevice, c->st));
  }
  int to_host(uint8_t* dst, uint64_t d, uint64_t len) {
    return c->check(cudaMemcpyAsync(dst, dev + d, len, cudaMemcpyDeviceToHost, c->st));
  }
  int record(int sl) { return c->check(cudaEventRecord(c->stage_ev[sl], c->st)); }
  int wait(int sl) { return c->check(cudaEventSynchronize(c->stage_ev[sl])); }
  void gather(const std::vector<StageHost>& h, uint8_t* slot) {
    std::vector<CopyJob> jobs;
    for (const StageHost& x : h) jobs.push_back(CopyJob{slot + x.slot_off, x.host, x.len});
    parallel_copy(jobs);
  }
  void scatter(const std::vector<StageHost>& h, const uint8_t* slot) {
    std::vector<CopyJob> jobs;
    for (const StageHost& x : h) jobs.push_back(CopyJob{x.host, slot + x.slot_off, x.len});
    parallel_copy(jobs);
  }
};

// run the ring over `fills` (upload: host -> dev, else dev -> host); on
// failure wait for the stream, so that no copy into or out of the ring
// outlives the call
int staged(gzgpu_ctx* c, const std::vector<StageFill>& fills, uint8_t* dev, bool upload) {
  if (!c->h_stage.ensure(2 * kStageSlot)) return GZGPU_DEVICE_ERROR;
  uint8_t* hb = reinterpret_cast<uint8_t*>(c->h_stage.p);
  uint8_t* const slots[2] = {hb, hb + kStageSlot};
  CudaStageOps ops{c, dev};
  const int rc = upload ? stage_upload(fills, slots, ops) : stage_download(fills, slots, ops);
  if (rc) cudaStreamSynchronize(c->st);
  return rc;
}

// host -> device copy of one stream into the context input buffer at `at`:
// page-locked caller memory by one DMA, pageable memory through the ring
int stage_input(gzgpu_ctx* c, const uint8_t* in, size_t n, uint64_t at) {
  if (!n) return kOk;
  if (host_pinned(in))
    return c->check(cudaMemcpyAsync(c->in.as<uint8_t>() + at, in, n, cudaMemcpyHostToDevice, c->st));
  const std::vector<StageSeg> segs{StageSeg{const_cast<uint8_t*>(in), at, n}};
  const std::vector<StageRun> runs{StageRun{at, at + n, 0, 1}};
  return staged(c, stage_plan(segs, runs), c->in.as<uint8_t>(), true);
}

// device -> host copy of `n` output bytes at `off`, the same way round; all
// of `out` is written when it returns
int deliver_output(gzgpu_ctx* c, uint8_t* out, uint64_t off, size_t n) {
  if (!n) return kOk;
  if (host_pinned(out)) {
    const int rc = c->check(cudaMemcpyAsync(out, c->cur_out + off, n, cudaMemcpyDeviceToHost, c->st));
    if (rc) cudaStreamSynchronize(c->st);
    return rc;
  }
  const std::vector<StageSeg> segs{StageSeg{out, off, n}};
  const std::vector<StageRun> runs{StageRun{off, off + n, 0, 1}};
  return staged(c, stage_plan(segs, runs), c->cur_out, false);
}

}  // namespace

namespace {

// one host stream through a job (caller holds c->mu): upload, decode, download
int decompress_host(gzgpu_ctx* c, const uint8_t* in, size_t in_len, uint8_t* out,
                    size_t out_cap, size_t* out_len) {
  cudaSetDevice(c->dev);
  reset_stats(c);
  int rc;
  if ((rc = c->check(c->in.ensure(in_len + kInputPad)))) return rc;
  cudaEventRecord(c->ev[0], c->st);
  if ((rc = stage_input(c, in, in_len, 0))) return rc;
  cudaMemsetAsync(c->in.as<uint8_t>() + in_len, 0, kInputPad, c->st);
  c->cur_in = c->in.as<uint8_t>();
  c->user_out = nullptr;
  std::vector<StreamSpec> S{{0, in_len}};
  std::vector<StreamOut> R;
  rc = c->job(S, R);
  if (rc != kOk) return rc;
  finish_stats(c);
  if (R[0].status != kOk) return R[0].status;
  *out_len = R[0].out_len;
  if (R[0].out_len > out_cap) return GZGPU_OUT_TOO_SMALL;
  cudaEvent_t t0 = c->ev[8], t1 = c->ev[9];
  cudaEventRecord(t0, c->st);
  if ((rc = deliver_output(c, out, R[0].out_off, R[0].out_len))) return rc;
  cudaEventRecord(t1, c->st);
  if ((rc = c->check(cudaStreamSynchronize(c->st)))) return rc;
  float t = 0;
  cudaEventElapsedTime(&t, t0, t1);
  c->stats.ms_d2h = t;
  t = 0;
  cudaEventElapsedTime(&t, c->ev[0], t1);
  c->stats.ms_total = t;
  return GZGPU_OK;
}

}  // namespace

int gzgpu_decompress(gzgpu_ctx* c, const uint8_t* in, size_t in_len, uint8_t* out,
                     size_t out_cap, size_t* out_len) {
  if (!c || !out_len || (!in && in_len) || (!out && out_cap)) return GZGPU_INVALID_ARGUMENT;
  *out_len = 0;
  if (in_len < 2 || in[0] != 0x1f || in[1] != 0x8b) return GZGPU_NOT_GZIP;
  std::lock_guard<std::mutex> g(c->mu);
  return decompress_host(c, in, in_len, out, out_cap, out_len);
}

int gzgpu_inflate_raw(gzgpu_ctx* c, const uint8_t* in, size_t in_len, uint8_t* out,
                      size_t out_cap, size_t* out_len) {
  if (!c || !out_len || (!in && in_len) || (!out && out_cap)) return GZGPU_INVALID_ARGUMENT;
  *out_len = 0;
  if (!in_len) return GZGPU_TRUNCATED;  // no final block
  std::lock_guard<std::mutex> g(c->mu);
  c->job_raw = true;
  const int rc = decompress_host(c, in, in_len, out, out_cap, out_len);
  c->job_raw = false;
  return rc;
}

int gzgpu_inflate_zlib(gzgpu_ctx* c, const uint8_t* in, size_t in_len, uint8_t* out,
                       size_t out_cap, size_t* out_len) {
  if (!c || !out_len || (!in && in_len) || (!out && out_cap)) return GZGPU_INVALID_ARGUMENT;
  *out_len = 0;
  // decompress_zlib_turbo (src/decompress/mod.rs:895-914): the DEFLATE data
  // between the 2-byte header and the 4-byte Adler-32, neither checked
  if (in_len < 6) return GZGPU_INVALID_ARGUMENT;
  return gzgpu_inflate_raw(c, in + 2, in_len - 6, out, out_cap, out_len);
}

int gzgpu_build_index(gzgpu_ctx* c, const uint8_t* in, size_t in_len, uint64_t interval_bytes,
                      uint8_t* index_out, size_t index_cap, size_t* index_len) {
  if (!c || !index_len || (!in && in_len) || (!index_out && index_cap)) return GZGPU_INVALID_ARGUMENT;
  *index_len = 0;
  // build_index (src/decompress/index.rs:55-80): gzip only, one member, and
  // not gzippy's multi-block format (its blocks are their own index)
  if (in_len < 18 || in[0] != 0x1f || in[1] != 0x8b) return GZGPU_INVALID_ARGUMENT;
  if (in[3] & 4) {
    const size_t xlen = in[10] | (in[11] << 8);
    for (size_t p = 12; p + 4 <= 12 + xlen && 12 + xlen <= in_len;) {
      if (in[p] == 'G' && in[p + 1] == 'Z') return GZGPU_INVALID_ARGUMENT;
      p += 4 + (in[p + 2] | (in[p + 3] << 8));
    }
  }
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  int rc;
  if ((rc = c->check(c->in.ensure(in_len + kInputPad)))) return rc;
  c->job_index = true;
  c->index_interval = interval_bytes;
  c->blk_need = 0;
  for (int attempt = 0; attempt < 2; attempt++) {
    reset_stats(c);
    cudaEventRecord(c->ev[0], c->st);
    if ((rc = stage_input(c, in, in_len, 0))) break;
    cudaMemsetAsync(c->in.as<uint8_t>() + in_len, 0, kInputPad, c->st);
    c->cur_in = c->in.as<uint8_t>();
    c->user_out = nullptr;
    std::vector<StreamSpec> S{{0, in_len}};
    std::vector<StreamOut> R;
    rc = c->job(S, R);
    if (rc != kOk) break;
    finish_stats(c);
    rc = c->index_status;
    if (rc != kPoolExhausted || !c->blk_need) break;  // else: again with the log sized to fit
  }
  c->job_index = false;
  if (rc != kOk) return rc == kPoolExhausted ? GZGPU_DEVICE_ERROR : rc;
  *index_len = c->index_bytes.size();
  if (c->index_bytes.size() > index_cap) return GZGPU_OUT_TOO_SMALL;
  memcpy(index_out, c->index_bytes.data(), c->index_bytes.size());
  return GZGPU_OK;
}

int gzgpu_decompress_device(gzgpu_ctx* c, const void* d_in, size_t in_len, void* d_out,
                            size_t out_cap, size_t* out_len) {
  if (!c || !out_len || (!d_in && in_len)) return GZGPU_INVALID_ARGUMENT;
  *out_len = 0;
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  reset_stats(c);
  if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15)
    return GZGPU_INVALID_ARGUMENT;  // the kernels use 16-byte vector access
  uint8_t magic[2] = {0, 0};
  if (in_len >= 2 && c->check(cudaMemcpy(magic, d_in, 2, cudaMemcpyDeviceToHost)))
    return GZGPU_DEVICE_ERROR;
  if (in_len < 2 || magic[0] != 0x1f || magic[1] != 0x8b) return GZGPU_NOT_GZIP;
  cudaEventRecord(c->ev[0], c->st);
  c->cur_in = reinterpret_cast<const uint8_t*>(d_in);
  c->user_out = reinterpret_cast<uint8_t*>(d_out);
  c->user_cap = out_cap;
  std::vector<StreamSpec> S{{0, in_len}};
  std::vector<StreamOut> R;
  int rc = c->job(S, R);
  c->user_out = nullptr;
  if (rc != kOk) return rc;
  finish_stats(c);
  if (R[0].status != kOk) return R[0].status;
  *out_len = R[0].out_len;
  if (R[0].out_len > out_cap) return GZGPU_OUT_TOO_SMALL;
  return GZGPU_OK;
}

int gzgpu_decompress_to_writer(gzgpu_ctx* c, const uint8_t* in, size_t in_len,
                               gzgpu_write_fn write, void* user, uint64_t* written) {
  if (!c || !write || (!in && in_len)) return GZGPU_INVALID_ARGUMENT;
  if (written) *written = 0;
  if (in_len < 2 || in[0] != 0x1f || in[1] != 0x8b) return GZGPU_NOT_GZIP;
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  reset_stats(c);
  int rc;
  if ((rc = c->check(c->in.ensure(in_len + kInputPad)))) return rc;
  cudaEventRecord(c->ev[0], c->st);
  if ((rc = stage_input(c, in, in_len, 0))) return rc;
  cudaMemsetAsync(c->in.as<uint8_t>() + in_len, 0, kInputPad, c->st);
  c->cur_in = c->in.as<uint8_t>();
  c->user_out = nullptr;
  std::vector<StreamSpec> S{{0, in_len}};
  std::vector<StreamOut> R;
  rc = c->job(S, R);
  if (rc != kOk) return rc;
  finish_stats(c);
  if (R[0].status != kOk) return R[0].status;
  // deliver in order through the pinned staging ring: the next piece
  // downloads while the writer consumes this one
  const size_t piece = kStageSlot;
  if (!c->h_stage.ensure(2 * piece)) return GZGPU_DEVICE_ERROR;
  uint8_t* hb = reinterpret_cast<uint8_t*>(c->h_stage.p);
  const uint64_t total = R[0].out_len;
  // piece i goes to half i % 2; piece i + 1 downloads while piece i is written
  auto issue = [&](uint64_t at) -> int {
    const int half = (int)((at / piece) & 1);
    const size_t k = (size_t)std::min<uint64_t>(piece, total - at);
    int e = c->check(cudaMemcpyAsync(hb + half * piece, c->cur_out + R[0].out_off + at, k,
                                     cudaMemcpyDeviceToHost, c->st));
    return e ? e : c->check(cudaEventRecord(c->stage_ev[half], c->st));
  };
  for (uint64_t at = 0; at < total && at < 2 * piece; at += piece)
    if ((rc = issue(at))) return rc;
  for (uint64_t at = 0; at < total; at += piece) {
    const int half = (int)((at / piece) & 1);
    const size_t k = (size_t)std::min<uint64_t>(piece, total - at);
    if ((rc = c->check(cudaEventSynchronize(c->stage_ev[half])))) return rc;
    if (write(user, hb + half * piece, k) != 0) {
      cudaStreamSynchronize(c->st);  // no download into the ring outlives the call
      return GZGPU_INVALID_ARGUMENT;
    }
    if (written) *written = at + k;
    if (at + 2 * piece < total && (rc = issue(at + 2 * piece))) return rc;
  }
  return GZGPU_OK;
}

int gzgpu_decompress_batch_device(gzgpu_ctx* c, const void* d_in, const uint64_t* in_offs,
                                  const uint64_t* in_lens, size_t n, void* d_out, size_t out_cap,
                                  uint64_t* out_offs, uint64_t* out_lens, int* statuses) {
  if (!c || (n && (!d_in || !in_offs || !in_lens || !out_offs || !out_lens || !statuses)))
    return GZGPU_INVALID_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15)
    return GZGPU_INVALID_ARGUMENT;  // the kernels use 16-byte vector access
  for (size_t i = 0; i < n; i++)
    if (in_offs[i] & 15) return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  reset_stats(c);
  std::vector<StreamSpec> S(n);
  for (size_t i = 0; i < n; i++) S[i] = StreamSpec{in_offs[i], in_lens[i]};
  cudaEventRecord(c->ev[0], c->st);
  c->cur_in = reinterpret_cast<const uint8_t*>(d_in);
  c->user_out = reinterpret_cast<uint8_t*>(d_out);
  c->user_cap = out_cap;
  std::vector<StreamOut> R;
  int rc = n ? c->job(S, R) : kOk;
  c->user_out = nullptr;
  if (rc != kOk) return rc;
  if (n) finish_stats(c);
  int all = GZGPU_OK;
  uint64_t total = 0;
  for (size_t i = 0; i < n; i++) {
    statuses[i] = R[i].status;
    out_offs[i] = R[i].out_off;
    out_lens[i] = R[i].status == kOk ? R[i].out_len : 0;
    if (R[i].status == kOk) total += R[i].out_len;
    if (statuses[i] != GZGPU_OK && statuses[i] != GZGPU_NOT_GZIP && all == GZGPU_OK) all = statuses[i];
  }
  if (all == GZGPU_OK && total > out_cap) return GZGPU_OUT_TOO_SMALL;
  return all;
}

int gzgpu_decompress_batch(gzgpu_ctx* c, const gzgpu_span* ins, size_t n, gzgpu_out* outs,
                           int* statuses) {
  if (!c || (n && (!ins || !outs || !statuses))) return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  reset_stats(c);
  uint64_t total = 0;
  for (size_t i = 0; i < n; i++) total += (ins[i].len + 15) & ~15ull;
  int rc;
  if ((rc = c->check(c->in.ensure(total + kInputPad)))) return rc;
  // pack the streams (16-byte aligned): direct ones by DMA from the caller's
  // page-locked buffers, the others through the staging ring
  std::vector<StreamSpec> S(n);
  std::vector<char> direct(n, 0);
  uint64_t at = 0;
  for (size_t i = 0; i < n; i++) {
    S[i] = StreamSpec{at, ins[i].len};
    direct[i] = ins[i].len >= kDirectBytes && host_pinned(ins[i].data);
    at += (ins[i].len + 15) & ~15ull;
  }
  // runs of consecutive staged streams: device ranges (alignment gaps
  // included) that the ring uploads piece by piece
  std::vector<StageSeg> segs;
  std::vector<StageRun> runs;
  for (size_t i = 0; i < n;) {
    if (direct[i]) {
      i++;
      continue;
    }
    const size_t s0 = segs.size();
    size_t j = i;
    for (; j < n && !direct[j]; j++)
      segs.push_back(StageSeg{const_cast<uint8_t*>(ins[j].data), S[j].off, ins[j].len});
    runs.push_back(StageRun{S[i].off, S[j - 1].off + S[j - 1].len, s0, segs.size()});
    i = j;
  }
  cudaEventRecord(c->ev[0], c->st);
  uint8_t* din = c->in.as<uint8_t>();
  for (size_t i = 0; i < n; i++)
    if (direct[i] && (rc = c->check(cudaMemcpyAsync(din + S[i].off, ins[i].data, ins[i].len,
                                                    cudaMemcpyHostToDevice, c->st))))
      return rc;
  if (!runs.empty() && (rc = staged(c, stage_plan(segs, runs), din, true))) return rc;
  cudaMemsetAsync(din + at, 0, kInputPad, c->st);
  c->cur_in = din;
  c->user_out = nullptr;
  std::vector<StreamOut> R;
  rc = c->job(S, R);
  if (rc != kOk) return rc;
  finish_stats(c);
  int all = GZGPU_OK;
  cudaEvent_t t0 = c->ev[8], t1 = c->ev[9];
  cudaEventRecord(t0, c->st);
  std::vector<char> deliver(n, 0);
  for (size_t i = 0; i < n; i++) {
    statuses[i] = R[i].status;
    outs[i].len = R[i].status == kOk ? R[i].out_len : 0;
    if (R[i].status == kOk && R[i].out_len > outs[i].cap) {
      statuses[i] = GZGPU_OUT_TOO_SMALL;
      outs[i].len = R[i].out_len;
    } else if (R[i].status == kOk && R[i].out_len) {
      deliver[i] = 1;
    }
    if (statuses[i] != GZGPU_OK && statuses[i] != GZGPU_NOT_GZIP && all == GZGPU_OK) all = statuses[i];
  }
  // outputs: large ones into page-locked caller memory by DMA; the rest in
  // runs contiguous on the device, downloaded through the staging ring
  std::vector<char> odirect(n, 0);
  for (size_t i = 0; i < n; i++)
    odirect[i] = deliver[i] && R[i].out_len >= kDirectBytes && host_pinned(outs[i].data);
  segs.clear();
  runs.clear();
  for (size_t i = 0; i < n;) {
    if (!deliver[i] || odirect[i]) {
      i++;
      continue;
    }
    const size_t s0 = segs.size();
    size_t j = i;
    do {
      segs.push_back(StageSeg{outs[j].data, R[j].out_off, R[j].out_len});
      j++;
    } while (j < n && deliver[j] && !odirect[j] && R[j].out_off == R[j - 1].out_off + R[j - 1].out_len);
    runs.push_back(StageRun{R[i].out_off, R[j - 1].out_off + R[j - 1].out_len, s0, segs.size()});
    i = j;
  }
  for (size_t i = 0; i < n; i++)
    if (odirect[i] && (rc = c->check(cudaMemcpyAsync(outs[i].data, c->cur_out + R[i].out_off,
                                                     R[i].out_len, cudaMemcpyDeviceToHost, c->st)))) {
      cudaStreamSynchronize(c->st);
      return rc;
    }
  if (!runs.empty() && (rc = staged(c, stage_plan(segs, runs), c->cur_out, false))) return rc;
  cudaEventRecord(t1, c->st);
  if ((rc = c->check(cudaStreamSynchronize(c->st)))) return rc;
  float t = 0;
  cudaEventElapsedTime(&t, t0, t1);
  c->stats.ms_d2h = t;
  t = 0;
  cudaEventElapsedTime(&t, c->ev[0], t1);
  c->stats.ms_total = t;
  return all;
}

int gzgpu_debug_find(gzgpu_ctx* c, const uint8_t* in, size_t in_len, const uint64_t* from,
                     const uint64_t* to, size_t n, uint64_t* lo, uint64_t* hi, int* valid) {
  if (!c || (!in && in_len) || (n && (!from || !to || !lo || !hi || !valid)))
    return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  int rc;
  if ((rc = c->check(c->in.ensure(in_len + kInputPad))) ||
      (rc = c->check(c->descs.ensure(sizeof(ChunkDesc) * (n + 1)))) ||
      (rc = c->check(c->spec.ensure(4 * (n + 1)))))
    return rc;
  cudaMemcpyAsync(c->in.p, in, in_len, cudaMemcpyHostToDevice, c->st);
  cudaMemsetAsync(c->in.as<uint8_t>() + in_len, 0, kInputPad, c->st);
  std::vector<ChunkDesc> d(n);
  std::vector<uint32_t> sp(n);
  for (size_t i = 0; i < n; i++) {
    d[i] = ChunkDesc{};
    d[i].guess_bit = d[i].start_bit = d[i].lo_bit = from[i];
    d[i].limit_bit = to[i];
    d[i].in_end = in_len;
    sp[i] = (uint32_t)i;
  }
  if (n) {
    cudaMemcpyAsync(c->descs.p, d.data(), sizeof(ChunkDesc) * n, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->spec.p, sp.data(), 4 * n, cudaMemcpyHostToDevice, c->st);
    if ((rc = c->check(launch_finder(c->in.as<uint8_t>(), c->descs.as<ChunkDesc>(),
                                     c->spec.as<uint32_t>(), (uint32_t)n, nullptr, c->st))))
      return rc;
    cudaMemcpyAsync(d.data(), c->descs.p, sizeof(ChunkDesc) * n, cudaMemcpyDeviceToHost, c->st);
  }
  if ((rc = c->check(cudaStreamSynchronize(c->st)))) return rc;
  for (size_t i = 0; i < n; i++) {
    valid[i] = (d[i].flags & kChunkValid) ? ((d[i].flags & kChunkSync) ? 2 : 1) : 0;
    lo[i] = d[i].lo_bit;
    hi[i] = d[i].start_bit;
  }
  return GZGPU_OK;
}

int gzgpu_debug_dyn_sync(gzgpu_ctx* c, const uint8_t* in, size_t in_len, const uint64_t* table_bit,
                         const uint64_t* from, const uint64_t* to, size_t n, uint64_t* out,
                         int* valid) {
  if (!c || (!in && in_len) || (n && (!table_bit || !from || !to || !out || !valid)))
    return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  int rc;
  if ((rc = c->check(c->in.ensure(in_len + kInputPad))) ||
      (rc = c->check(c->descs.ensure(sizeof(ChunkDesc) * (2 * n + 1)))) ||
      (rc = c->check(c->spec.ensure(4 * (n + 1)))))
    return rc;
  cudaMemcpyAsync(c->in.p, in, in_len, cudaMemcpyHostToDevice, c->st);
  cudaMemsetAsync(c->in.as<uint8_t>() + in_len, 0, kInputPad, c->st);
  // each range is a piece after a parent whose start is the block's header
  std::vector<ChunkDesc> d(2 * n);
  std::vector<uint32_t> pieces(n);
  for (size_t i = 0; i < n; i++) {
    ChunkDesc& p = d[2 * i];
    p = ChunkDesc{};
    p.start_bit = p.lo_bit = p.guess_bit = table_bit[i];
    p.limit_bit = from[i];
    p.in_end = in_len;
    p.flags = kChunkValid;
    ChunkDesc& q = d[2 * i + 1];
    q = ChunkDesc{};
    q.start_bit = q.lo_bit = q.guess_bit = from[i];
    q.limit_bit = to[i];
    q.in_end = in_len;
    q.flags = kChunkPiece;
    pieces[i] = (uint32_t)(2 * i + 1);
  }
  if (n) {
    cudaMemcpyAsync(c->descs.p, d.data(), sizeof(ChunkDesc) * 2 * n, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->spec.p, pieces.data(), 4 * n, cudaMemcpyHostToDevice, c->st);
    if ((rc = c->check(launch_dyn_sync(c->in.as<uint8_t>(), c->descs.as<ChunkDesc>(),
                                       c->spec.as<uint32_t>(), (uint32_t)n, nullptr, c->st))))
      return rc;
    cudaMemcpyAsync(d.data(), c->descs.p, sizeof(ChunkDesc) * 2 * n, cudaMemcpyDeviceToHost, c->st);
  }
  if ((rc = c->check(cudaStreamSynchronize(c->st)))) return rc;
  for (size_t i = 0; i < n; i++) {
    const ChunkDesc& q = d[2 * i + 1];
    valid[i] = (q.flags & kChunkValid) ? 1 : 0;
    out[i] = valid[i] ? q.start_bit : 0;
  }
  return GZGPU_OK;
}

int gzgpu_debug_decode(gzgpu_ctx* c, const uint8_t* in, size_t in_len, const uint64_t* start,
                       const uint64_t* stop, const int* flags, size_t n, uint16_t* entries,
                       size_t cap_per, uint64_t* res, const uint64_t* table_bit) {
  if (!c || (!in && in_len) || (n && (!start || !stop || !flags || !res)))
    return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(c->mu);
  cudaSetDevice(c->dev);
  int rc;
  uint64_t pages_needed = n * 64 + in_len / 4096 + 64;
  if ((rc = c->check(c->in.ensure(in_len + kInputPad))) ||
      (rc = c->check(c->descs.ensure(sizeof(ChunkDesc) * (n + 1)))) ||
      (rc = c->check(c->results.ensure(sizeof(ChunkResult) * (n + 1)))) ||
      (rc = c->check(c->work.ensure(4 * (n + 1)))) || (rc = c->check(c->counters.ensure(64))) ||
      (rc = c->check(c->pages.ensure(pages_needed * kPageEntries * 2))) ||
      (rc = c->check(c->owner.ensure(4 * pages_needed))) ||
      (rc = c->check(c->seq.ensure(4 * pages_needed))))
    return rc;
  cudaMemcpyAsync(c->in.p, in, in_len, cudaMemcpyHostToDevice, c->st);
  cudaMemsetAsync(c->in.as<uint8_t>() + in_len, 0, kInputPad, c->st);
  std::vector<ChunkDesc> d(n);
  std::vector<uint32_t> wl(n);
  for (size_t i = 0; i < n; i++) {
    d[i] = ChunkDesc{};
    d[i].start_bit = d[i].lo_bit = d[i].guess_bit = d[i].limit_bit = start[i];
    d[i].stop_lo = stop[i];
    d[i].abort_bit = kNoStop;
    d[i].next = kNoChunk;
    d[i].in_end = in_len;
    d[i].flags = kChunkValid | ((flags[i] & 1) ? kChunkMemberFirst : 0u) |
                 ((flags[i] & 2) ? kChunkSync : 0u);
    d[i].table_bit = table_bit ? table_bit[i] : 0;
    wl[i] = (uint32_t)i;
  }
  // a chunk followed by a sync start may stop at it mid-block
  for (size_t i = 0; i + 1 < n; i++)
    if (d[i + 1].flags & kChunkSync) d[i].next = (uint32_t)(i + 1);
  uint32_t nn = (uint32_t)n;
  cudaMemsetAsync(c->counters.p, 0, 64, c->st);
  if (n) {
    cudaMemcpyAsync(c->descs.p, d.data(), sizeof(ChunkDesc) * n, cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->work.p, wl.data(), 4 * n, cudaMemcpyHostToDevice, c->st);
  }
  cudaMemcpyAsync(c->counters.as<uint32_t>() + 1, &nn, 4, cudaMemcpyHostToDevice, c->st);
  c->cur_in = c->in.as<uint8_t>();
  c->job_sync = false;
  for (size_t i = 0; i < n; i++) c->job_sync |= (d[i].flags & kChunkSync) != 0;
  if ((rc = c->check(c->launch_decode(c->counters.as<uint32_t>() + 1)))) return rc;
  std::vector<ChunkResult> r(n);
  uint32_t used = 0;
  if (n) cudaMemcpyAsync(r.data(), c->results.p, sizeof(ChunkResult) * n, cudaMemcpyDeviceToHost, c->st);
  cudaMemcpyAsync(&used, c->counters.as<uint32_t>() + 2, 4, cudaMemcpyDeviceToHost, c->st);
  if ((rc = c->check(cudaStreamSynchronize(c->st)))) return rc;
  const uint64_t cap = std::min<uint64_t>(c->pages.cap / (kPageEntries * 2),
                                          std::min(c->owner.cap, c->seq.cap) / 4);
  used = (uint32_t)std::min<uint64_t>(used, cap);
  std::vector<uint32_t> own(used), sq(used);
  if (used) {
    cudaMemcpy(own.data(), c->owner.p, 4 * used, cudaMemcpyDeviceToHost);
    cudaMemcpy(sq.data(), c->seq.p, 4 * used, cudaMemcpyDeviceToHost);
  }
  for (size_t i = 0; i < n; i++) {
    uint64_t* o = res + 7 * i;
    o[0] = r[i].end_bit;
    o[1] = r[i].out_len;
    o[2] = r[i].marker_end;
    o[3] = r[i].n_blocks;
    o[4] = (uint64_t)(int64_t)r[i].status;
    o[5] = r[i].final_block;
    o[6] = r[i].sync_end;
  }
  if (entries) {
    for (uint32_t p = 0; p < used; p++) {
      uint32_t cid = own[p];
      if (cid >= n || r[cid].status != kOk || (sq[p] >> kGenShift) != r[cid].gen) continue;
      uint64_t q0 = (uint64_t)(sq[p] & kSeqMask) * kPageEntries;
      if (q0 >= r[cid].out_len || q0 >= cap_per) continue;
      uint64_t k = std::min<uint64_t>({(uint64_t)kPageEntries, r[cid].out_len - q0, cap_per - q0});
      cudaMemcpy(entries + cid * cap_per + q0, c->pages.as<uint16_t>() + (size_t)p * kPageEntries,
                 2 * k, cudaMemcpyDeviceToHost);
    }
  }
  return GZGPU_OK;
}

int gzgpu_debug_last_chunks(gzgpu_ctx* c, void* descs, void* results, size_t cap, size_t* n) {
  if (!c || !n) return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(c->mu);
  *n = c->last_descs.size();
  size_t k = std::min(cap, c->last_descs.size());
  if (descs && k) memcpy(descs, c->last_descs.data(), k * sizeof(ChunkDesc));
  if (results && k) memcpy(results, c->last_results.data(), k * sizeof(ChunkResult));
  return GZGPU_OK;
}

int gzgpu_get_stats(gzgpu_ctx* c, gzgpu_stats* out) {
  if (!c || !out) return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(c->mu);
  *out = c->stats;
  return GZGPU_OK;
}

}  // extern "C"
