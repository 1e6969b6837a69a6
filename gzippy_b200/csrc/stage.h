// stage.h -- copies between pageable host buffers and device memory through
// a fixed pinned ring of two slots.
//
// The staged streams of a batch form runs: device byte ranges [dev0, dev1)
// that hold one or more streams (with the alignment gaps between them).  A
// plan cuts the runs into pieces of at most one slot and packs consecutive
// pieces into slot fills; a fill is one host gather or scatter (memcpy, in
// parallel) plus one DMA per piece.  Fills alternate between the two slots,
// so the host copies of one overlap the DMA of the other, and the pinned
// memory is allocated once: no page-locking or unpinning on the serving path,
// where either can stall every stream of the device.
//
// Plain C++ (no CUDA types): the executor takes the device operations as a
// callback object, so the same code runs against memcpy on the CPU.
#pragma once
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace gzgpu {

constexpr uint64_t kStageSlot = 32ull << 20;  // bytes per slot; the ring holds two

struct StageSeg {  // one stream's bytes
  uint8_t* host;   // caller buffer: read by uploads, written by downloads
  uint64_t dev;    // byte offset on the device
  uint64_t len;
};

struct StageRun {  // device range [dev0, dev1) holding segs[seg0, seg1), in device order
  uint64_t dev0, dev1;
  size_t seg0, seg1;
};

struct StageDma {
  uint64_t slot_off, dev, len;
};

struct StageHost {
  uint8_t* host;
  uint64_t slot_off, len;
};

struct StageFill {
  std::vector<StageDma> dma;
  std::vector<StageHost> host;
};

// Cut the runs into fills of at most slot_bytes (a multiple of 16); pieces
// start at 16-byte aligned slot offsets.
inline std::vector<StageFill> stage_plan(const std::vector<StageSeg>& segs,
                                         const std::vector<StageRun>& runs,
                                         uint64_t slot_bytes = kStageSlot) {
  std::vector<StageFill> fills;
  uint64_t used = slot_bytes;  // the first piece opens a fill
  for (const StageRun& r : runs) {
    size_t s = r.seg0;
    for (uint64_t x = r.dev0; x < r.dev1;) {
      used = (used + 15) & ~15ull;
      if (used >= slot_bytes) {
        fills.emplace_back();
        used = 0;
      }
      const uint64_t y = std::min(r.dev1, x + (slot_bytes - used));
      StageFill& f = fills.back();
      f.dma.push_back(StageDma{used, x, y - x});
      while (s < r.seg1 && segs[s].dev + segs[s].len <= x) s++;
      for (size_t k = s; k < r.seg1 && segs[k].dev < y; k++) {
        const uint64_t a = std::max(x, segs[k].dev);
        const uint64_t b = std::min(y, segs[k].dev + segs[k].len);
        if (b > a) f.host.push_back(StageHost{segs[k].host + (a - segs[k].dev), used + (a - x), b - a});
      }
      used += y - x;
      x = y;
    }
  }
  return fills;
}

// Ops: int to_dev(uint64_t dev, const uint8_t* src, uint64_t len);
//      int to_host(uint8_t* dst, uint64_t dev, uint64_t len);
//      int record(int slot);  int wait(int slot);   (0 = ok)
//      void gather(const std::vector<StageHost>&, uint8_t* slot);   host -> slot
//      void scatter(const std::vector<StageHost>&, const uint8_t* slot);   slot -> host
// Fill i uses slot i % 2.

// Uploads: a slot is refilled only after its previous DMA has finished.
// The last DMAs are still in flight on return (ordered before later work on
// the same stream).
template <class Ops>
int stage_upload(const std::vector<StageFill>& fills, uint8_t* const slots[2], Ops& ops) {
  for (size_t i = 0; i < fills.size(); i++) {
    const int sl = (int)(i & 1);
    int rc;
    if (i >= 2 && (rc = ops.wait(sl))) return rc;
    ops.gather(fills[i].host, slots[sl]);
    for (const StageDma& d : fills[i].dma)
      if ((rc = ops.to_dev(d.dev, slots[sl] + d.slot_off, d.len))) return rc;
    if ((rc = ops.record(sl))) return rc;
  }
  return 0;
}

// Downloads: two fills' DMAs are in flight while the host scatters the
// older one; all of the host buffers are written on return.
template <class Ops>
int stage_download(const std::vector<StageFill>& fills, uint8_t* const slots[2], Ops& ops) {
  auto issue = [&](size_t i) -> int {
    const int sl = (int)(i & 1);
    int rc;
    for (const StageDma& d : fills[i].dma)
      if ((rc = ops.to_host(slots[sl] + d.slot_off, d.dev, d.len))) return rc;
    return ops.record(sl);
  };
  int rc;
  for (size_t i = 0; i < fills.size() && i < 2; i++)
    if ((rc = issue(i))) return rc;
  for (size_t i = 0; i < fills.size(); i++) {
    const int sl = (int)(i & 1);
    if ((rc = ops.wait(sl))) return rc;
    ops.scatter(fills[i].host, slots[sl]);
    if (i + 2 < fills.size() && (rc = issue(i + 2))) return rc;
  }
  return 0;
}

}  // namespace gzgpu
