// CPU check of the pinned staging ring (gzippy_b200/csrc/stage.h).
//
// The device is a byte array and the CUDA stream a FIFO of deferred copies:
// a copy runs only when a wait() on a later event of its slot, or the final
// stream sync, drains the FIFO up to it.  That models the asynchrony the ring
// relies on: a gather into a slot whose earlier DMA has not run yet, or a
// scatter of a slot whose DMA has not run yet, shows up as a hazard or as
// wrong bytes.  Random layouts of streams (sizes from 0 to several slots,
// alignment gaps, runs broken by direct streams) are uploaded and downloaded
// with small slots and compared byte for byte; bytes outside the streams
// must stay untouched.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <random>
#include <vector>

#include "../gzippy_b200/csrc/stage.h"

using namespace gzgpu;

namespace {

struct Op {
  int kind;  // 0 = to_dev, 1 = to_host, 2 = event
  uint8_t* host;
  uint64_t dev, len;
  int slot;
};

struct FakeStream {
  std::vector<uint8_t>& dev;
  uint8_t* slots[2];
  uint64_t slot_bytes;
  std::deque<Op> fifo;
  int hazards = 0;

  bool in_slot(const uint8_t* p, int sl) const { return p >= slots[sl] && p < slots[sl] + slot_bytes; }
  void run(const Op& o) {
    if (o.kind == 0) memcpy(dev.data() + o.dev, o.host, o.len);
    if (o.kind == 1) memcpy(o.host, dev.data() + o.dev, o.len);
  }
  void drain_to_last_event(int sl) {
    size_t last = fifo.size();
    for (size_t i = 0; i < fifo.size(); i++)
      if (fifo[i].kind == 2 && fifo[i].slot == sl) last = i;
    if (last == fifo.size()) return;
    for (size_t i = 0; i <= last; i++) {
      run(fifo.front());
      fifo.pop_front();
    }
  }
  void sync() {
    while (!fifo.empty()) {
      run(fifo.front());
      fifo.pop_front();
    }
  }
  bool pending_on(int sl) const {
    for (const Op& o : fifo)
      if (o.kind != 2 && in_slot(o.host, sl)) return true;
    return false;
  }
  int slot_of(const uint8_t* p) const { return in_slot(p, 0) ? 0 : in_slot(p, 1) ? 1 : -1; }

  int to_dev(uint64_t d, const uint8_t* src, uint64_t len) {
    fifo.push_back(Op{0, const_cast<uint8_t*>(src), d, len, -1});
    return 0;
  }
  int to_host(uint8_t* dst, uint64_t d, uint64_t len) {
    fifo.push_back(Op{1, dst, d, len, -1});
    return 0;
  }
  int record(int sl) {
    fifo.push_back(Op{2, nullptr, 0, 0, sl});
    return 0;
  }
  int wait(int sl) {
    drain_to_last_event(sl);
    return 0;
  }
  void gather(const std::vector<StageHost>& h, uint8_t* slot) {
    if (pending_on(slot_of(slot))) hazards++;
    for (const StageHost& x : h) memcpy(slot + x.slot_off, x.host, x.len);
  }
  void scatter(const std::vector<StageHost>& h, const uint8_t* slot) {
    if (pending_on(slot_of(slot))) hazards++;
    for (const StageHost& x : h) memcpy(x.host, slot + x.slot_off, x.len);
  }
};

struct Layout {
  std::vector<StageSeg> segs;
  std::vector<StageRun> runs;
  uint64_t dev_bytes = 0;
};

// streams at 16-byte aligned device offsets; some are "direct" (not staged),
// which breaks runs exactly as the batch path does
Layout make_layout(std::mt19937_64& rng, std::vector<std::vector<uint8_t>>& bufs, uint64_t slot) {
  Layout L;
  const int n = 1 + (int)(rng() % 40);
  uint64_t at = 0;
  bool in_run = false;
  for (int i = 0; i < n; i++) {
    uint64_t len;
    switch (rng() % 4) {
      case 0: len = rng() % 16; break;
      case 1: len = rng() % 300; break;
      case 2: len = rng() % (slot + 100); break;
      default: len = rng() % (3 * slot + 7); break;
    }
    const bool direct = rng() % 5 == 0;
    if (!direct) {
      bufs.emplace_back(len + 32, 0xA5);  // 16-byte canaries each side
      L.segs.push_back(StageSeg{bufs.back().data() + 16, at, len});
      if (!in_run) L.runs.push_back(StageRun{at, at, L.segs.size() - 1, L.segs.size() - 1});
      L.runs.back().dev1 = at + len;
      L.runs.back().seg1 = L.segs.size();
      in_run = true;
    } else {
      in_run = false;
    }
    at += (len + 15) & ~15ull;
    if (rng() % 7 == 0) at += 16 * (rng() % 4);  // extra gap inside a run
  }
  L.dev_bytes = at + 64;
  return L;
}

}  // namespace

int main() {
  std::mt19937_64 rng(20261204);
  int fails = 0, cases = 0;
  for (int t = 0; t < 3000; t++) {
    const uint64_t slot = 16 * (1 + rng() % 64);  // 16 B .. 1 KiB slots
    std::vector<std::vector<uint8_t>> bufs;
    bufs.reserve(64);
    Layout L = make_layout(rng, bufs, slot);
    std::vector<uint8_t> ring(2 * slot);
    uint8_t* slots[2] = {ring.data(), ring.data() + slot};
    std::vector<StageFill> fills = stage_plan(L.segs, L.runs, slot);
    // every piece fits its slot, at an aligned offset
    for (const StageFill& f : fills)
      for (const StageDma& d : f.dma)
        if (d.slot_off % 16 || d.slot_off + d.len > slot) fails++;

    // upload: host streams with random bytes -> device
    for (StageSeg& s : L.segs)
      for (uint64_t k = 0; k < s.len; k++) s.host[k] = (uint8_t)rng();
    std::vector<uint8_t> dev(L.dev_bytes, 0x5A);
    std::vector<uint8_t> want = dev;
    for (const StageSeg& s : L.segs) memcpy(want.data() + s.dev, s.host, s.len);
    // gaps inside a run are copied too (their slot bytes are unspecified)
    std::vector<char> covered(L.dev_bytes, 0);
    for (const StageRun& r : L.runs)
      for (uint64_t k = r.dev0; k < r.dev1; k++) covered[k] = 1;
    std::vector<char> is_seg(L.dev_bytes, 0);
    for (const StageSeg& s : L.segs)
      for (uint64_t k = 0; k < s.len; k++) is_seg[s.dev + k] = 1;
    FakeStream up{dev, {slots[0], slots[1]}, slot};
    stage_upload(fills, slots, up);
    up.sync();
    for (uint64_t k = 0; k < L.dev_bytes; k++) {
      if (is_seg[k] && dev[k] != want[k]) { fails++; break; }
      if (!covered[k] && dev[k] != 0x5A) { fails++; break; }
    }
    fails += up.hazards;

    // download: device random -> host streams
    for (uint8_t& b : dev) b = (uint8_t)rng();
    for (std::vector<uint8_t>& b : bufs) std::fill(b.begin(), b.end(), 0xA5);
    FakeStream down{dev, {slots[0], slots[1]}, slot};
    stage_download(fills, slots, down);
    if (!down.fifo.empty()) fails++;  // all delivered on return
    fails += down.hazards;
    for (const StageSeg& s : L.segs) {
      if (memcmp(s.host, dev.data() + s.dev, s.len) != 0) fails++;
      for (int k = 1; k <= 16; k++)
        if (s.host[-k] != 0xA5 || s.host[s.len + k - 1] != 0xA5) { fails++; break; }
    }
    cases++;
  }
  printf("%d cases, %d failures\n", cases, fails);
  return fails ? 1 : 0;
}
