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
//   * each admitted request is issued on the least recently used of S streams
//     (H2D copy, execute, D2H copy, frees), so requests that arrive while
//     others run overlap with them on the GPU; the copies go in pieces of
//     8 MiB so that a small request's copy need not wait behind a whole large
//     transfer on a copy engine.
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
  Clock::time_point t_submit, t_done;
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
  std::thread dispatcher, completer;
  uint64_t next_id = 1;
  std::vector<double> latencies_ms;
  Clock::time_point t_first, t_last;
  uint64_t completed = 0, failed = 0;
  int max_inflight_seen = 0;
  // plan-instance churn: creations (and their wall time) and evictions
  uint64_t plans_created = 0, plans_evicted = 0;
  double create_ms_total = 0, create_ms_max = 0;
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
cudaError_t copy_chunked(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t st) {
  for (size_t off = 0; off < bytes; off += kCopyChunk) {
    const size_t n = bytes - off < kCopyChunk ? bytes - off : kCopyChunk;
    const cudaError_t e = cudaMemcpyAsync(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                                          n, kind, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

void dispatcher_loop(shafft_sm100_server_s* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    if (s->queue.empty()) {
      s->cv_queue.wait_for(lk, std::chrono::milliseconds(20));
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
      if (s->used + hneed > s->budget && s->inflight.empty() && s->building.empty()) {
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
      s->cv_queue.wait_for(lk, std::chrono::microseconds(200));
      continue;
    }
    const size_t need = 2 * r->bytes;
    s->used += need;
    // least recently used stream
    int si = 0;
    for (int i = 1; i < s->nstreams; ++i)
      if (s->stream_last[i] < s->stream_last[si]) si = i;
    s->stream_last[si] = Clock::now();
    r->inst = inst;
    r->stream = si;
    cudaStream_t st = s->streams[si];
    lk.unlock();
    cudaError_t e = cudaMallocFromPoolAsync(&r->d_in, r->bytes, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&r->d_out, r->bytes, s->pool, st);
    if (e == cudaSuccess) e = copy_chunked(r->d_in, r->host_in, r->bytes, cudaMemcpyHostToDevice, st);
    int xrc = 0;
    if (e == cudaSuccess)
      xrc = shafft_sm100_execute(inst->plan, r->d_in, r->d_out, r->direction, r->scale, st);
    if (e == cudaSuccess && !xrc)
      e = copy_chunked(r->host_out, r->d_out, r->bytes, cudaMemcpyDeviceToHost, st);
    if (r->d_in) cudaFreeAsync(r->d_in, st);
    if (r->d_out) cudaFreeAsync(r->d_out, st);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(r->ev, st);
    lk.lock();
    if (e != cudaSuccess || xrc) {
      r->status = xrc ? xrc : sfail(SHAFFT_SM100_ECUDA, "issue: %s", cudaGetErrorString(e));
      cudaStreamSynchronize(st);
      r->done = true;
      r->t_done = Clock::now();
      s->used -= need;
      inst->users--;
      s->failed++;
      s->cv_done.notify_all();
      continue;
    }
    s->inflight.push_back(r);
    s->max_inflight_seen = std::max<int>(s->max_inflight_seen, (int)s->inflight.size());
  }
}

void completer_loop(shafft_sm100_server_s* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop || !s->inflight.empty()) {
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
        s->latencies_ms.push_back(
            std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        if (s->completed == 1) s->t_first = r->t_submit;
        s->t_last = r->t_done;
      }
      cudaEventDestroy(r->ev);
      r->ev = nullptr;
      s->used -= 2 * r->bytes;
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
  for (int i = 0; e == cudaSuccess && i < streams; ++i) {
    cudaStream_t st = nullptr;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    s->streams.push_back(st);
    s->stream_last.push_back(Clock::now());
  }
  if (e != cudaSuccess) {
    for (auto st : s->streams)
      if (st) cudaStreamDestroy(st);
    if (s->pool) cudaMemPoolDestroy(s->pool);
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
  std::vector<double> v = s->latencies_ms;
  std::sort(v.begin(), v.end());
  auto pct = [&](double q) { return v.empty() ? 0.0 : v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
  const double span = s->completed ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0;
  snprintf(buf, buflen,
           "{\"completed\":%llu,\"failed\":%llu,\"p50_ms\":%.4f,\"p99_ms\":%.4f,\"max_ms\":%.4f,"
           "\"throughput_per_s\":%.3f,\"max_inflight\":%d,\"resident_plan_bytes\":%zu,\"streams\":%d,"
           "\"plans_created\":%llu,\"plans_evicted\":%llu,\"plan_create_ms_total\":%.3f,"
           "\"plan_create_ms_max\":%.3f}",
           (unsigned long long)s->completed, (unsigned long long)s->failed, pct(0.5), pct(0.99),
           v.empty() ? 0.0 : v.back(), span > 0 ? s->completed / span : 0.0, s->max_inflight_seen,
           s->plan_bytes, s->nstreams, (unsigned long long)s->plans_created,
           (unsigned long long)s->plans_evicted, s->create_ms_total, s->create_ms_max);
  return 0;
}

int shafft_sm100_server_reset_stats(shafft_sm100_server s) {
  if (!s) return sfail(SHAFFT_SM100_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->latencies_ms.clear();
  s->completed = s->failed = 0;
  s->max_inflight_seen = 0;
  s->plans_created = s->plans_evicted = 0;
  s->create_ms_total = s->create_ms_max = 0;
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
  delete s;
  return 0;
}

}  // extern "C"
