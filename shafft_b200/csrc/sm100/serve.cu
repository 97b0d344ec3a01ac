// Serving form: a request loop with continuous admission.
//
// Clients submit C2C transforms (shape, precision, direction, scale, host
// input and output buffers) from any thread.  A dispatcher thread admits
// requests in arrival order as soon as their device memory fits the budget
// and a plan instance of their shape is free; a request whose shape has no
// free instance asks a builder thread for one and lets the requests behind it
// (up to kScanWindow) go first, so plan creation (device allocations, table
// kernels, a synchronisation: tens of ms for large shapes) overlaps the
// transforms instead of stalling the queue.  Memory admission stays in
// arrival order: a request that does not fit the budget holds back the ones
// behind it.
//   * device input/output buffers come from the server's own stream-ordered
//     memory pool (cudaMallocFromPoolAsync / cudaFreeAsync), so freeing is
//     ordered after the work; it reuses only blocks whose frees completed,
//     so no request's stream waits on another's;
//   * plans are kept resident per shape; requests of one shape that overlap
//     share its instance when the plan has no scratch or control state
//     (plan_shareable), and get instances of their own otherwise; idle
//     instances are evicted oldest-first when the budget needs their memory;
//   * each admitted request is issued on the one of S streams with the
//     fewest bytes in flight (H2D copy, execute, D2H copy, frees), so that it
//     does not queue behind a large request, and requests that arrive while
//     others run overlap with them on the GPU; the copies go in pieces of
//     8 MiB so that a small request's copy need not wait behind a whole large
//     transfer on a copy engine; requests with buffers of 256 MiB or more
//     copy in turn with each other, one per direction at a time.
// A completion thread polls the per-request events, releases the budget and
// the plan instance, stamps the completion time and wakes waiters.  Latency
// is completion time minus submission time; statistics report p50 / p99.
// With the same plan arithmetic a request's result is bit-identical whether
// it ran alone or in a mix (tested).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/shafft_sm100.h"
#include "launch.h"

namespace shafft_sm100 {
namespace {

int sfail(int code, const char* fmt, ...) {
  char msg[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt, ap);
  va_end(ap);
  return report_error(code, msg);
}

using Clock = std::chrono::steady_clock;

struct PlanInst {
  shafft_sm100_plan plan = nullptr;
  int users = 0;        // requests in flight on this instance
  bool shared = false;  // plan_shareable: any number of users at once
  size_t bytes = 0;
  Clock::time_point last_used;
};

struct Request {
  uint64_t id = 0;
  std::vector<int64_t> dims;
  int precision = 0, direction = 0;
  double scale = 1.0;
  const void* host_in = nullptr;
  void* host_out = nullptr;
  size_t bytes = 0;  // one buffer
  Clock::time_point t_submit, t_issue, t_done;
  // in flight
  void* d_in = nullptr;
  void* d_out = nullptr;
  cudaEvent_t ev = nullptr;
  PlanInst* inst = nullptr;
  int stream = -1;
  int status = 0;
  bool done = false;
};

}  // namespace
}  // namespace shafft_sm100

using namespace shafft_sm100;

struct shafft_sm100_server_s {
  size_t budget = 0, used = 0;
  int nstreams = 0;
  std::vector<cudaStream_t> streams;
  std::vector<Clock::time_point> stream_last;
  std::vector<size_t> stream_bytes;  // device bytes of the requests in flight on each stream
  cudaMemPool_t pool = nullptr;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_queue, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::vector<std::shared_ptr<Request>> inflight;
  std::map<uint64_t, std::shared_ptr<Request>> all;
  std::map<std::string, std::vector<std::unique_ptr<PlanInst>>> plans;
  size_t plan_bytes = 0;
  std::atomic<bool> stop{false};
  std::atomic<bool> dispatch_done{false};  // the dispatcher has issued its last request
  std::thread dispatcher, completer;
  uint64_t next_id = 1;
  std::vector<double> latencies_ms;
  std::vector<double> admit_ms;  // submission to the start of issue, per completed request
  Clock::time_point t_first, t_last;
  uint64_t completed = 0, failed = 0;
  int max_inflight_seen = 0;
  // plan-instance churn: creations (and their wall time) and evictions
  uint64_t plans_created = 0, plans_evicted = 0;
  double create_ms_total = 0, create_ms_max = 0;
  // wall time of the dispatcher's CUDA calls for one request (allocation,
  // copies, transform launches) or one round of pump steps: the longest
  double issue_ms_max = 0;
  // background plan creation: shapes waiting for an instance (one build in
  // flight per shape)
  struct BuildJob {
    std::string key;
    std::vector<int64_t> dims;
    int precision;
  };
  std::deque<BuildJob> build_q;
  std::map<std::string, int> building;
  std::condition_variable cv_build;
  std::thread builder;
  // Large requests (kLargeCopy bytes a buffer or more) copy one at a time in
  // each direction, in admission order: each waits for the previous large
  // request's copy in the same direction (these events, recorded after it).
  cudaEvent_t large_h2d = nullptr, large_d2h = nullptr;
  // Copies of the requests issued whole (below kLargeCopy) not yet known to
  // be done, one event each, per direction (dispatcher thread only).  The
  // copy engines do not interleave another stream's copy with a large copy
  // that keeps being fed (measured on B200: a 1 MiB copy waited 13 ms behind
  // a 906 MiB copy fed two 8 MiB pieces at a time), so a pump holds its next
  // piece back while one of these is pending.
  std::deque<cudaEvent_t> small_h2d, small_d2h;
};

namespace {

std::string plan_key(const Request& r) {
  std::string k = r.precision ? "z" : "c";
  for (int64_t d : r.dims) k += ":" + std::to_string(d);
  return k;
}

constexpr size_t kScanWindow = 64;  // queued requests the dispatcher looks past a plan-blocked one

// caller holds s->mu: an instance of r's shape that can take another user
// (its user count raised), or null after asking the builder for one (unless
// a build of that shape runs)
PlanInst* free_instance(shafft_sm100_server_s* s, const Request& r) {
  const std::string key = plan_key(r);
  auto it = s->plans.find(key);
  if (it != s->plans.end())
    for (auto& p : it->second)
      if (p->users == 0 || p->shared) {
        p->users++;
        p->last_used = Clock::now();
        return p.get();
      }
  if (!s->building.count(key)) {
    s->building[key] = 1;
    s->build_q.push_back(shafft_sm100_server_s::BuildJob{key, r.dims, r.precision});
    s->cv_build.notify_one();
  }
  return nullptr;
}

// Creates the plan instances the dispatcher asks for, with the lock released
// while a plan is built so that admissions and completions keep flowing.  A
// shape whose plan cannot be created fails its queued requests.
void builder_loop(shafft_sm100_server_s* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    if (s->build_q.empty()) {
      s->cv_build.wait_for(lk, std::chrono::milliseconds(20));
      continue;
    }
    const shafft_sm100_server_s::BuildJob job = s->build_q.front();
    s->build_q.pop_front();
    lk.unlock();
    shafft_sm100_plan pl = nullptr;
    const auto t0 = Clock::now();
    const int rc = shafft_sm100_plan_create_nd(&pl, (int)job.dims.size(), job.dims.data(), job.precision);
    const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    lk.lock();
    s->plans_created++;
    s->create_ms_total += ms;
    s->create_ms_max = std::max(s->create_ms_max, ms);
    s->building.erase(job.key);
    if (rc) {
      for (auto it = s->queue.begin(); it != s->queue.end();) {
        if (plan_key(**it) == job.key) {
          (*it)->status = rc;
          (*it)->done = true;
          (*it)->t_done = Clock::now();
          s->failed++;
          it = s->queue.erase(it);
        } else {
          ++it;
        }
      }
      s->cv_done.notify_all();
    } else {
      auto inst = std::make_unique<PlanInst>();
      inst->plan = pl;
      inst->shared = plan_shareable(pl);
      inst->bytes = shafft_sm100_plan_device_bytes(pl);
      inst->last_used = Clock::now();
      s->plan_bytes += inst->bytes;
      s->used += inst->bytes;
      s->plans[job.key].push_back(std::move(inst));
    }
    s->cv_queue.notify_all();
  }
}

// caller holds s->mu: unlink idle plan instances, oldest first, until the
// resident plans leave room for `need` bytes, keeping the instances of the
// shape `keep_key` (the request the room is made for would otherwise lose the
// plan it waits for and ask for it again).  Buffers of requests in flight
// are not counted: they come back as those requests complete, so waiting for
// them is cheaper than destroying and later re-creating plans.  The unlinked plans are returned in `dead` and
// destroyed by the caller after it drops the lock (cudaFree synchronises the
// device, which must not happen while completions wait for the lock).
void evict_idle(shafft_sm100_server_s* s, size_t need, const std::string& keep_key,
                std::vector<shafft_sm100_plan>& dead) {
  while (s->plan_bytes + need > s->budget) {
    PlanInst* victim = nullptr;
    std::string vkey;
    for (auto& kv : s->plans) {
      if (kv.first == keep_key) continue;  // the waiting request's own shape
      for (auto& p : kv.second)
        if (p->users == 0 && (!victim || p->last_used < victim->last_used)) {
          victim = p.get();
          vkey = kv.first;
        }
    }
    if (!victim) return;
    auto& vec = s->plans[vkey];
    for (size_t i = 0; i < vec.size(); ++i)
      if (vec[i].get() == victim) {
        dead.push_back(victim->plan);
        s->plans_evicted++;
        s->plan_bytes -= victim->bytes;
        s->used -= victim->bytes;
        vec.erase(vec.begin() + i);
        break;
      }
    if (vec.empty()) s->plans.erase(vkey);
  }
}

// Host<->device copies of a request in pieces of at most kCopyChunk bytes:
// a small request's copy on another stream can then start after one piece
// of a large transfer already queued on the copy engine instead of after the
// whole transfer.
constexpr size_t kCopyChunk = size_t(8) << 20;
// a request whose buffers are this large copies in turn with the other large
// ones (two overlapping large copies would both take twice as long; in turn,
// the first one is done at full speed and the second no later)
constexpr size_t kLargeCopy = size_t(256) << 20;
cudaError_t copy_chunked(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
  for (size_t off = 0; off < bytes; off += kCopyChunk) {
    const size_t n = bytes - off < kCopyChunk ? bytes - off : kCopyChunk;
    const cudaError_t e = cudaMemcpyAsync(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                                          n, kind, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The copies of a large request are fed to the copy engines a few 8 MiB
// pieces at a time (a "pump"), so that a small request's copy queued
// meanwhile waits for at most kPumpDepth pieces, not for the whole transfer.
// Large requests also take each direction in turn, in admission order.
// States: 0 waits for the host-to-device lane, 1 issues its pieces, 2 waits
// for the device-to-host lane (the transform is issued), 3 issues those
// pieces, 4 done (the request's completion event is recorded).
constexpr int kPumpDepth = 2;
constexpr std::chrono::microseconds kPumpHold(2000);
struct Pump {
  std::shared_ptr<Request> r;
  cudaStream_t st = nullptr;
  int si = 0;
  int state = 0;
  size_t off = 0;
  cudaEvent_t ev[kPumpDepth] = {};
  int head = 0, count = 0;
  bool holding = false;  // a piece held back for small copies since hold_since
  Clock::time_point hold_since;
};

// Drop the finished copies at the front of `q`; true while one is pending.
bool copies_pending(std::deque<cudaEvent_t>& q) {
  while (!q.empty()) {
    const cudaError_t e = cudaEventQuery(q.front());
    if (e == cudaErrorNotReady) return true;
    cudaEventDestroy(q.front());  // done (or failed: its request reports that)
    q.pop_front();
  }
  return false;
}

// Advance one pump as far as it can go now; `lane_h2d` / `lane_d2h` say
// whether an earlier pump holds that lane.  Returns a CUDA error, or
// cudaSuccess (also when it had to wait).
cudaError_t pump_step(shafft_sm100_server_s* s, Pump& p, bool lane_h2d, bool lane_d2h) {
  Request& r = *p.r;
  while (p.count > 0) {  // retire finished pieces
    const cudaError_t q = cudaEventQuery(p.ev[p.head]);
    if (q == cudaErrorNotReady) break;
    if (q != cudaSuccess) return q;
    p.head = (p.head + 1) % kPumpDepth;
    p.count--;
  }
  cudaError_t e = cudaSuccess;
  for (;;) {
    if (p.state == 0) {
      if (lane_h2d) return cudaSuccess;
      e = cudaStreamWaitEvent(p.st, s->large_h2d, 0);
      if (e != cudaSuccess) return e;
      p.state = 1;
      p.off = 0;
    } else if (p.state == 2) {
      if (lane_d2h) return cudaSuccess;
      e = cudaStreamWaitEvent(p.st, s->large_d2h, 0);
      if (e != cudaSuccess) return e;
      p.state = 3;
      p.off = 0;
    } else if (p.state == 1 || p.state == 3) {
      if (p.off < r.bytes) {
        if (p.count == kPumpDepth) return cudaSuccess;  // wait for a piece to finish
        // hold the piece back for pending small copies, for at most
        // kPumpHold at a stretch so that a steady stream of small requests
        // cannot starve the large one
        if (copies_pending(p.state == 1 ? s->small_h2d : s->small_d2h)) {
          const auto now = Clock::now();
          if (!p.holding) {
            p.holding = true;
            p.hold_since = now;
          }
          if (now - p.hold_since < kPumpHold) return cudaSuccess;
        }
        p.holding = false;
        const size_t n = std::min(kCopyChunk, r.bytes - p.off);
        e = p.state == 1 ? cudaMemcpyAsync(static_cast<char*>(r.d_in) + p.off,
                                           static_cast<const char*>(r.host_in) + p.off, n,
                                           cudaMemcpyHostToDevice, p.st)
                         : cudaMemcpyAsync(static_cast<char*>(r.host_out) + p.off,
                                           static_cast<const char*>(r.d_out) + p.off, n,
                                           cudaMemcpyDeviceToHost, p.st);
        if (e == cudaSuccess) e = cudaEventRecord(p.ev[(p.head + p.count) % kPumpDepth], p.st);
        if (e != cudaSuccess) return e;
        p.count++;
        p.off += n;
      } else if (p.state == 1) {
        e = cudaEventRecord(s->large_h2d, p.st);
        if (e != cudaSuccess) return e;
        const int xrc = shafft_sm100_execute(r.inst->plan, r.d_in, r.d_out, r.direction, r.scale, p.st);
        if (xrc) {
          r.status = xrc;  // the library's own status; the caller reports it
          return cudaErrorUnknown;
        }
        p.state = 2;
      } else {
        e = cudaEventRecord(s->large_d2h, p.st);
        if (e == cudaSuccess) e = cudaFreeAsync(r.d_in, p.st);
        if (e == cudaSuccess) r.d_in = nullptr;
        if (e == cudaSuccess) e = cudaFreeAsync(r.d_out, p.st);
        if (e == cudaSuccess) r.d_out = nullptr;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r.ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(r.ev, p.st);
        if (e != cudaSuccess) return e;
        p.state = 4;
        return cudaSuccess;
      }
    } else {
      return cudaSuccess;
    }
  }
}

// caller holds s->mu: a request that failed while being issued
void fail_issue(shafft_sm100_server_s* s, Request& r, cudaError_t e) {
  if (!r.status) r.status = sfail(SHAFFT_SM100_ECUDA, "issue: %s", cudaGetErrorString(e));
  cudaStreamSynchronize(s->streams[r.stream]);
  r.done = true;
  r.t_done = Clock::now();
  s->used -= 2 * r.bytes;
  s->stream_bytes[r.stream] -= 2 * r.bytes;
  r.inst->users--;
  s->failed++;
  s->cv_done.notify_all();
}

void dispatcher_loop(shafft_sm100_server_s* s) {
  cudaSetDevice(s->device);
  std::vector<Pump> pumps;  // large requests whose copies are being fed
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop || !pumps.empty()) {
    if (!pumps.empty()) {
      const auto t0 = Clock::now();
      lk.unlock();
      // in admission order: a pump waits for a lane held or awaited by an earlier one
      bool h2d_busy = false, d2h_busy = false;
      std::vector<cudaError_t> errs(pumps.size(), cudaSuccess);
      for (size_t i = 0; i < pumps.size(); ++i) {
        errs[i] = pump_step(s, pumps[i], h2d_busy, d2h_busy);
        const int st = pumps[i].state;
        h2d_busy |= (st <= 1);
        d2h_busy |= (st == 2 || st == 3);
      }
      lk.lock();
      s->issue_ms_max = std::max(s->issue_ms_max, std::chrono::duration<double, std::milli>(Clock::now() - t0).count());
      for (size_t i = pumps.size(); i-- > 0;) {
        Pump& p = pumps[i];
        if (errs[i] == cudaSuccess && p.state != 4) continue;
        if (errs[i] != cudaSuccess) {
          if (p.r->d_in) cudaFreeAsync(p.r->d_in, p.st);
          if (p.r->d_out) cudaFreeAsync(p.r->d_out, p.st);
          fail_issue(s, *p.r, errs[i]);
        } else {
          s->inflight.push_back(p.r);
          s->max_inflight_seen = std::max<int>(s->max_inflight_seen, (int)s->inflight.size());
        }
        for (cudaEvent_t ev : p.ev)
          if (ev) cudaEventDestroy(ev);
        pumps.erase(pumps.begin() + i);
      }
    }
    const auto nap = pumps.empty() ? std::chrono::microseconds(20000) : std::chrono::microseconds(50);
    if (s->stop) {
      s->cv_queue.wait_for(lk, nap);
      continue;
    }
    if (s->queue.empty()) {
      s->cv_queue.wait_for(lk, nap);
      continue;
    }
    {
      std::shared_ptr<Request> head = s->queue.front();
      const size_t hneed = 2 * head->bytes;
      if (s->plan_bytes + hneed > s->budget) {
        std::vector<shafft_sm100_plan> dead;
        evict_idle(s, hneed, plan_key(*head), dead);
        if (!dead.empty()) {
          lk.unlock();
          for (auto pl : dead) shafft_sm100_plan_destroy(pl);
          lk.lock();
          continue;  // the queue may have changed meanwhile
        }
      }
      if (s->used + hneed > s->budget && s->inflight.empty() && pumps.empty() && s->building.empty()) {
        // can never fit: fail it instead of blocking the queue
        s->queue.pop_front();
        head->status = sfail(SHAFFT_SM100_EALLOC, "request needs %zu bytes, budget %zu", hneed, s->budget);
        head->done = true;
        head->t_done = Clock::now();
        s->failed++;
        s->cv_done.notify_all();
        continue;
      }
    }
    // the first request, in arrival order, that fits the budget and has a
    // free plan instance; a request that does not fit stops the scan
    std::shared_ptr<Request> r;
    PlanInst* inst = nullptr;
    size_t pos = 0;
    for (auto it = s->queue.begin(); it != s->queue.end() && pos < kScanWindow; ++it, ++pos) {
      if (s->used + 2 * (*it)->bytes > s->budget) break;
      inst = free_instance(s, **it);
      if (inst) {
        r = *it;
        s->queue.erase(it);
        break;
      }
    }
    if (!r) {
      s->cv_queue.wait_for(lk, pumps.empty() ? std::chrono::microseconds(200) : std::chrono::microseconds(50));
      continue;
    }
    const size_t need = 2 * r->bytes;
    s->used += need;
    // the stream with the fewest bytes of requests still in flight (the
    // least recently used among equals): a request issued behind a large
    // one on the same stream would wait for all of it
    int si = 0;
    for (int i = 1; i < s->nstreams; ++i)
      if (s->stream_bytes[i] < s->stream_bytes[si] ||
          (s->stream_bytes[i] == s->stream_bytes[si] && s->stream_last[i] < s->stream_last[si]))
        si = i;
    s->stream_last[si] = Clock::now();
    s->stream_bytes[si] += need;
    r->inst = inst;
    r->stream = si;
    cudaStream_t st = s->streams[si];
    const auto t_issue = Clock::now();
    r->t_issue = t_issue;
    lk.unlock();
    cudaError_t e = cudaMallocFromPoolAsync(&r->d_in, r->bytes, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&r->d_out, r->bytes, s->pool, st);
    if (e == cudaSuccess && r->bytes >= kLargeCopy) {
      // a large request: its copies go through a pump
      Pump p;
      p.r = r;
      p.st = st;
      p.si = si;
      for (int k = 0; k < kPumpDepth && e == cudaSuccess; ++k)
        e = cudaEventCreateWithFlags(&p.ev[k], cudaEventDisableTiming);
      if (e == cudaSuccess) {
        lk.lock();
        s->issue_ms_max =
            std::max(s->issue_ms_max, std::chrono::duration<double, std::milli>(Clock::now() - t_issue).count());
        pumps.push_back(p);
        continue;
      }
      for (cudaEvent_t ev : p.ev)
        if (ev) cudaEventDestroy(ev);
    }
    // a copy that a pump should let through first: an event after it
    auto mark = [&](std::deque<cudaEvent_t>& q) {
      if (pumps.empty() || e != cudaSuccess) return;
      cudaEvent_t ev = nullptr;
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventRecord(ev, st);
      if (e == cudaSuccess)
        q.push_back(ev);
      else if (ev)
        cudaEventDestroy(ev);
    };
    if (e == cudaSuccess) e = copy_chunked(r->d_in, r->host_in, r->bytes, cudaMemcpyHostToDevice, st);
    mark(s->small_h2d);
    int xrc = 0;
    if (e == cudaSuccess)
      xrc = shafft_sm100_execute(inst->plan, r->d_in, r->d_out, r->direction, r->scale, st);
    if (e == cudaSuccess && !xrc)
      e = copy_chunked(r->host_out, r->d_out, r->bytes, cudaMemcpyDeviceToHost, st);
    if (!xrc) mark(s->small_d2h);
    if (r->d_in) cudaFreeAsync(r->d_in, st);
    if (r->d_out) cudaFreeAsync(r->d_out, st);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(r->ev, st);
    lk.lock();
    s->issue_ms_max = std::max(s->issue_ms_max, std::chrono::duration<double, std::milli>(Clock::now() - t_issue).count());
    if (e != cudaSuccess || xrc) {
      if (xrc) r->status = xrc;
      fail_issue(s, *r, e);
      continue;
    }
    s->inflight.push_back(r);
    s->max_inflight_seen = std::max<int>(s->max_inflight_seen, (int)s->inflight.size());
  }
  s->dispatch_done = true;
}

void completer_loop(shafft_sm100_server_s* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->dispatch_done || !s->inflight.empty()) {
    bool any = false;
    for (size_t i = 0; i < s->inflight.size();) {
      auto r = s->inflight[i];
      const cudaError_t q = cudaEventQuery(r->ev);
      if (q == cudaErrorNotReady) {
        ++i;
        continue;
      }
      r->t_done = Clock::now();
      if (q != cudaSuccess) {
        r->status = sfail(SHAFFT_SM100_ECUDA, "request %llu: %s", (unsigned long long)r->id,
                          cudaGetErrorString(q));
        s->failed++;
      } else {
        s->completed++;
        s->admit_ms.push_back(std::chrono::duration<double, std::milli>(r->t_issue - r->t_submit).count());
        s->latencies_ms.push_back(
            std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        if (s->completed == 1) s->t_first = r->t_submit;
        s->t_last = r->t_done;
      }
      cudaEventDestroy(r->ev);
      r->ev = nullptr;
      s->used -= 2 * r->bytes;
      s->stream_bytes[r->stream] -= 2 * r->bytes;
      r->inst->users--;
      r->inst->last_used = Clock::now();
      r->done = true;
      s->inflight.erase(s->inflight.begin() + i);
      any = true;
    }
    if (any) {
      s->cv_done.notify_all();
      s->cv_queue.notify_all();
    }
    lk.unlock();
    std::this_thread::sleep_for(std::chrono::microseconds(any ? 0 : 20));
    lk.lock();
  }
}

}  // namespace

extern "C" {

int shafft_sm100_server_create(shafft_sm100_server* out, size_t budget_bytes, int streams) {
  if (!out || budget_bytes == 0 || streams < 1 || streams > 64)
    return sfail(SHAFFT_SM100_EINVAL, "bad server arguments");
  *out = nullptr;
  auto* s = new (std::nothrow) shafft_sm100_server_s();
  if (!s) return sfail(SHAFFT_SM100_EALLOC, "host allocation failed");
  s->budget = budget_bytes;
  s->nstreams = streams;
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) {
    // the server's own pool: its settings do not leak into the process's
    // default pool
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    e = cudaMemPoolCreate(&s->pool, &props);
  }
  if (e == cudaSuccess) {
    uint64_t keep = UINT64_MAX;  // keep freed blocks cached in the pool
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e == cudaSuccess) {
    // A request's buffers may reuse blocks whose frees have completed, but
    // never a block still in use by another stream's request: with internal
    // dependencies allowed, the pool would make a small request's stream
    // wait for a large request on another stream to finish.
    int no = 0;
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->large_h2d, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->large_d2h, cudaEventDisableTiming);
  for (int i = 0; e == cudaSuccess && i < streams; ++i) {
    cudaStream_t st = nullptr;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    s->streams.push_back(st);
    s->stream_last.push_back(Clock::now());
    s->stream_bytes.push_back(0);
  }
  if (e != cudaSuccess) {
    for (auto st : s->streams)
      if (st) cudaStreamDestroy(st);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->large_h2d) cudaEventDestroy(s->large_h2d);
    if (s->large_d2h) cudaEventDestroy(s->large_d2h);
    delete s;
    return sfail(SHAFFT_SM100_ECUDA, "server set-up: %s", cudaGetErrorString(e));
  }
  // Grow the memory pool to the budget now (or to what the device can
  // spare): a pool that first grows while requests run maps gigabytes of
  // new memory on the request path, which showed as second-long stalls when
  // the number of requests in flight first rose.  The pool keeps the memory
  // (release threshold above), and later requests carve their buffers out
  // of it.
  for (size_t want = budget_bytes; want >= (size_t(1) << 30); want /= 2) {
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, want, s->pool, s->streams[0]) == cudaSuccess) {
      cudaFreeAsync(p, s->streams[0]);
      cudaStreamSynchronize(s->streams[0]);
      break;
    }
    cudaGetLastError();
  }
  s->dispatcher = std::thread(dispatcher_loop, s);
  s->completer = std::thread(completer_loop, s);
  s->builder = std::thread(builder_loop, s);
  *out = s;
  return 0;
}

int shafft_sm100_server_submit(shafft_sm100_server s, int ndim, const int64_t* dims, int precision,
                               int direction, double scale, const void* host_in, void* host_out,
                               uint64_t* id) {
  if (!s || !dims || ndim < 1 || !host_in || !host_out || !id)
    return sfail(SHAFFT_SM100_EINVAL, "bad request");
  if (precision != 0 && precision != 1) return sfail(SHAFFT_SM100_EINVAL, "bad precision");
  auto r = std::make_shared<Request>();
  r->dims.assign(dims, dims + ndim);
  int64_t n = 1;
  for (int a = 0; a < ndim; ++a) {
    if (dims[a] < 1) return sfail(SHAFFT_SM100_EINVAL, "bad dims");
    n *= dims[a];
  }
  r->precision = precision;
  r->direction = direction;
  r->scale = scale;
  r->host_in = host_in;
  r->host_out = host_out;
  r->bytes = (size_t)n * (precision ? 16 : 8);
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(s->mu);
  r->id = s->next_id++;
  *id = r->id;
  s->all[r->id] = r;
  s->queue.push_back(r);
  s->cv_queue.notify_one();
  return 0;
}

int shafft_sm100_server_wait(shafft_sm100_server s, uint64_t id, double* latency_ms) {
  if (!s) return sfail(SHAFFT_SM100_EINVAL, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return sfail(SHAFFT_SM100_EINVAL, "unknown request %llu", (unsigned long long)id);
  auto r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  const int st = r->status;
  s->all.erase(id);
  return st;
}

int shafft_sm100_server_stats(shafft_sm100_server s, char* buf, int buflen) {
  if (!s || !buf || buflen <= 0) return sfail(SHAFFT_SM100_EINVAL, "bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> v = s->latencies_ms, va = s->admit_ms;
  std::sort(va.begin(), va.end());
  const double admit_p99 = va.empty() ? 0.0 : va[std::min(va.size() - 1, (size_t)(0.99 * (va.size() - 1) + 0.5))];
  std::sort(v.begin(), v.end());
  auto pct = [&](double q) { return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
  const double span = s->completed ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0;
  snprintf(buf, buflen,
           "{\"completed\":%llu,\"failed\":%llu,\"p50_ms\":%.4f,\"p99_ms\":%.4f,\"max_ms\":%.4f,"
           "\"throughput_per_s\":%.3f,\"max_inflight\":%d,\"resident_plan_bytes\":%zu,\"streams\":%d,"
           "\"plans_created\":%llu,\"plans_evicted\":%llu,\"plan_create_ms_total\":%.3f,"
           "\"plan_create_ms_max\":%.3f,\"issue_ms_max\":%.3f,\"admit_wait_p99_ms\":%.4f}",
           (unsigned long long)s->completed, (unsigned long long)s->failed, pct(0.5), pct(0.99),
           v.empty() ? 0.0 : v.back(), span > 0 ? s->completed / span : 0.0, s->max_inflight_seen,
           s->plan_bytes, s->nstreams, (unsigned long long)s->plans_created,
           (unsigned long long)s->plans_evicted, s->create_ms_total, s->create_ms_max, s->issue_ms_max, admit_p99);
  return 0;
}

int shafft_sm100_server_reset_stats(shafft_sm100_server s) {
  if (!s) return sfail(SHAFFT_SM100_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->latencies_ms.clear();
  s->admit_ms.clear();
  s->completed = s->failed = 0;
  s->max_inflight_seen = 0;
  s->plans_created = s->plans_evicted = 0;
  s->create_ms_total = s->create_ms_max = 0;
  s->issue_ms_max = 0;
  return 0;
}

int shafft_sm100_server_destroy(shafft_sm100_server s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_queue.notify_all();
    s->cv_build.notify_all();
  }
  s->dispatcher.join();
  s->completer.join();
  s->builder.join();
  for (auto st : s->streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (auto& kv : s->plans)
    for (auto& p : kv.second) shafft_sm100_plan_destroy(p->plan);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  cudaEventDestroy(s->large_h2d);
  cudaEventDestroy(s->large_d2h);
  for (auto* q : {&s->small_h2d, &s->small_d2h})
    for (cudaEvent_t ev : *q) cudaEventDestroy(ev);
  delete s;
  return 0;
}

}  // extern "C"
