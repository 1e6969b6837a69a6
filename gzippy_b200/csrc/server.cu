// server.cu -- continuous-batching decompression service (gzgpu_server_*).
//
// No counterpart in the reference, which decodes one buffer per call.  Built
// only on the public entry points of gzgpu.h:
//   * a request queue (FIFO) fed by gzgpu_submit from any thread;
//   * `lanes` worker threads, each owning a gzgpu_ctx: its own CUDA stream
//     and device buffers (input, chunk tables, page pool, output), which stay
//     allocated from one batch to the next;
//   * admission against a device-memory budget: a request is charged its
//     compressed size + 3 x its output capacity (output bytes and the u16
//     pages the decoder writes) + 1 MiB, from admission until it completes;
//   * batching: a free lane takes the request at the front of the queue; a
//     large one (compressed size >= large_bytes) runs alone, otherwise the
//     lane merges the small requests behind it (up to max_batch_bytes of
//     input) into one gzgpu_decompress_batch job, i.e. one persistent decode
//     launch.  `small_lanes` lanes take only small requests (passing large
//     ones by), so small requests do not wait while large ones hold every
//     lane; their streams have the device's greatest priority, so their
//     thread blocks are scheduled before the large jobs' pending ones.  Lanes run concurrently, so requests that arrive while others
//     are on the GPU start as soon as a lane and budget free up, and their
//     kernels overlap with the batches already running.
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gzgpu.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kNoStatus = -1;

struct Request {
  uint64_t id;
  const uint8_t* in;
  size_t in_len;
  uint8_t* out;
  size_t out_cap;
  size_t charge;  // budget bytes held from admission to completion
  Clock::time_point t_submit, t_admit, t_done;
  int status = GZGPU_PENDING;
  size_t out_len = 0;
  bool done = false;
};

}  // namespace

struct gzgpu_server {
  gzgpu_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work;  // lanes wait for admissible work
  std::condition_variable cv_done;  // pollers wait for completions
  std::deque<Request*> queue;
  std::unordered_map<uint64_t, Request*> live;  // submitted, not yet collected
  uint64_t next_id = 1;
  size_t budget_used = 0;
  bool stop = false;
  std::vector<gzgpu_ctx*> ctxs;
  std::vector<std::thread> lanes;
  gzgpu_server_stats st{};

  bool admissible() const {
    if (queue.empty()) return false;
    const Request* r = queue.front();
    return budget_used + r->charge <= cfg.budget_bytes;
  }
  // a small request (in FIFO order among the small ones) that fits the budget
  bool admissible_small() const {
    for (const Request* r : queue)
      if (r->in_len < cfg.large_bytes) return budget_used + r->charge <= cfg.budget_bytes;
    return false;
  }
  // pop the small requests at the front of the small ones (caller holds mu);
  // the lanes reserved for small requests take these, passing large ones by
  void take_small_batch(std::vector<Request*>& b) {
    b.clear();
    size_t in_total = 0;
    const auto now = Clock::now();
    for (auto it = queue.begin(); it != queue.end();) {
      Request* r = *it;
      if (r->in_len >= cfg.large_bytes) {
        ++it;
        continue;
      }
      if (!b.empty() && in_total + r->in_len > cfg.max_batch_bytes) break;
      if (budget_used + r->charge > cfg.budget_bytes) break;
      it = queue.erase(it);
      budget_used += r->charge;
      r->t_admit = now;
      b.push_back(r);
      in_total += r->in_len;
      if (b.size() >= cfg.max_batch_requests) break;
    }
  }

  // pop the next batch (caller holds mu)
  void take_batch(std::vector<Request*>& b) {
    b.clear();
    size_t in_total = 0;
    const auto now = Clock::now();
    while (!queue.empty()) {
      Request* r = queue.front();
      const bool large = r->in_len >= cfg.large_bytes;
      if (!b.empty() && (large || in_total + r->in_len > cfg.max_batch_bytes)) break;
      if (budget_used + r->charge > cfg.budget_bytes) break;
      queue.pop_front();
      budget_used += r->charge;
      r->t_admit = now;
      b.push_back(r);
      in_total += r->in_len;
      if (large || b.size() >= cfg.max_batch_requests) break;
    }
  }

  void lane_main(int lane) {
    gzgpu_ctx* ctx = ctxs[lane];
    const bool small_only = lane < cfg.small_lanes;
    std::vector<Request*> batch;
    std::vector<gzgpu_span> spans;
    std::vector<gzgpu_out> outs;
    std::vector<int> statuses;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || (small_only ? admissible_small() : admissible()); });
        if (stop) return;
        if (small_only) take_small_batch(batch);
        else take_batch(batch);
        st.batches++;
        st.in_flight += batch.size();
      }
      spans.resize(batch.size());
      outs.resize(batch.size());
      statuses.assign(batch.size(), kNoStatus);
      for (size_t i = 0; i < batch.size(); i++) {
        spans[i] = gzgpu_span{batch[i]->in, batch[i]->in_len};
        outs[i] = gzgpu_out{batch[i]->out, batch[i]->out_cap, 0};
      }
      int rc = gzgpu_decompress_batch(ctx, spans.data(), spans.size(), outs.data(), statuses.data());
      const auto now = Clock::now();
      {
        std::lock_guard<std::mutex> lk(mu);
        for (size_t i = 0; i < batch.size(); i++) {
          Request* r = batch[i];
          // a job that failed as a whole set no per-request status
          r->status = statuses[i] == kNoStatus ? rc : statuses[i];
          r->out_len = outs[i].len;
          r->t_done = now;
          r->done = true;
          budget_used -= r->charge;
          st.completed++;
          st.out_bytes += r->status == GZGPU_OK ? r->out_len : 0;
          st.in_bytes += r->in_len;
        }
        st.in_flight -= batch.size();
      }
      cv_done.notify_all();
      cv_work.notify_all();  // budget freed: any lane may admit now
    }
  }
};

extern "C" {

int gzgpu_server_create(gzgpu_server** out, const gzgpu_server_config* cfg) {
  if (!out) return GZGPU_INVALID_ARGUMENT;
  *out = nullptr;
  gzgpu_server* s = new (std::nothrow) gzgpu_server();
  if (!s) return GZGPU_DEVICE_ERROR;
  if (cfg) s->cfg = *cfg;
  if (!s->cfg.budget_bytes) s->cfg.budget_bytes = 120ull << 30;
  if (s->cfg.lanes <= 0) s->cfg.lanes = 4;
  if (s->cfg.small_lanes == 0) s->cfg.small_lanes = s->cfg.lanes >= 2 ? 1 : 0;
  if (s->cfg.small_lanes < 0 || s->cfg.small_lanes >= s->cfg.lanes) s->cfg.small_lanes = 0;
  if (!s->cfg.max_batch_bytes) s->cfg.max_batch_bytes = 256ull << 20;
  if (!s->cfg.max_batch_requests) s->cfg.max_batch_requests = 4096;
  if (!s->cfg.large_bytes) s->cfg.large_bytes = 32ull << 20;
  for (int i = 0; i < s->cfg.lanes; i++) {
    gzgpu_config c{};
    c.device = s->cfg.device;
    c.autotune = s->cfg.autotune;
    // small requests' kernels go ahead of large ones' pending blocks
    c.high_priority = i < s->cfg.small_lanes;
    gzgpu_ctx* ctx = nullptr;
    int rc = gzgpu_create(&ctx, &c);
    if (rc != GZGPU_OK) {
      for (gzgpu_ctx* x : s->ctxs) gzgpu_destroy(x);
      delete s;
      return rc;
    }
    s->ctxs.push_back(ctx);
  }
  for (int i = 0; i < s->cfg.lanes; i++) s->lanes.emplace_back([s, i] { s->lane_main(i); });
  *out = s;
  return GZGPU_OK;
}

void gzgpu_server_destroy(gzgpu_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (std::thread& t : s->lanes) t.join();
  for (gzgpu_ctx* c : s->ctxs) gzgpu_destroy(c);
  for (auto& kv : s->live) delete kv.second;
  delete s;
}

int gzgpu_submit(gzgpu_server* s, const uint8_t* in, size_t in_len, uint8_t* out, size_t out_cap,
                 uint64_t* ticket) {
  if (!s || !ticket || (!in && in_len) || (!out && out_cap)) return GZGPU_INVALID_ARGUMENT;
  Request* r = new (std::nothrow) Request();
  if (!r) return GZGPU_DEVICE_ERROR;
  r->in = in;
  r->in_len = in_len;
  r->out = out;
  r->out_cap = out_cap;
  r->charge = in_len + 3 * out_cap + (1u << 20);
  if (r->charge > s->cfg.budget_bytes) {
    delete r;
    return GZGPU_OVER_BUDGET;
  }
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    s->live[r->id] = r;
    s->queue.push_back(r);
    s->st.submitted++;
  }
  *ticket = r->id;
  // every lane: a lane reserved for small requests does not take a large one,
  // so waking only one could leave the request queued with a general lane idle
  s->cv_work.notify_all();
  return GZGPU_OK;
}

int gzgpu_poll(gzgpu_server* s, uint64_t ticket, int wait_ms, size_t* out_len,
               gzgpu_request_times* times) {
  if (!s) return GZGPU_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->live.find(ticket);
  if (it == s->live.end()) return GZGPU_INVALID_ARGUMENT;
  Request* r = it->second;
  if (!r->done && wait_ms != 0) {
    auto ready = [&] { return r->done; };
    if (wait_ms < 0) s->cv_done.wait(lk, ready);
    else s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  }
  if (!r->done) return GZGPU_PENDING;
  if (out_len) *out_len = r->out_len;
  if (times) {
    auto ms = [](Clock::duration d) { return std::chrono::duration<double, std::milli>(d).count(); };
    times->queue_ms = ms(r->t_admit - r->t_submit);
    times->total_ms = ms(r->t_done - r->t_submit);
  }
  const int status = r->status;
  s->live.erase(it);
  delete r;
  return status;
}

int gzgpu_server_get_stats(gzgpu_server* s, gzgpu_server_stats* out) {
  if (!s || !out) return GZGPU_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->queued = s->queue.size();
  out->budget_used = s->budget_used;
  return GZGPU_OK;
}

}  // extern "C"
