// context.cu — per-device context, per-thread streams, last-error, scratch memory.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"

namespace zkb {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

const char *last_error() { return g_last_error.c_str(); }

static std::mutex g_ctx_mu;
static std::vector<std::unique_ptr<DeviceContext>> g_ctx;

int current_context(DeviceContext **out) {
  int dev = 0;
  ZKB_CHECK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if ((int)g_ctx.size() <= dev) g_ctx.resize(dev + 1);
  if (!g_ctx[dev]) {
    auto c = std::make_unique<DeviceContext>();
    c->device = dev;
    ZKB_CHECK_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, dev));
    // Keep freed scratch in the pool: commits of the same shape reuse it without
    // returning memory to the driver between calls.  A block freed on one stream is reused
    // on another only once its free has completed (or the stream already waits for it):
    // reuse through an inserted dependency would make, e.g., one engine job's FRI phase
    // wait for every kernel queued on another job's stream.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
      int no = 0;
      cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    }
    g_ctx[dev] = std::move(c);
  }
  *out = g_ctx[dev].get();
  return ZKB_OK;
}

namespace {
struct ThreadStreams {
  std::vector<cudaStream_t> per_dev;
  ~ThreadStreams() {
    // Streams are released with the process; destroying them at thread exit
    // could race with work the thread enqueued and never synchronised.
  }
};
thread_local ThreadStreams t_streams;
}  // namespace

cudaStream_t thread_stream() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  if ((int)t_streams.per_dev.size() <= dev) t_streams.per_dev.resize(dev + 1, nullptr);
  if (!t_streams.per_dev[dev]) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    t_streams.per_dev[dev] = s;
  }
  return t_streams.per_dev[dev];
}

// --------------------------------------------------------------- profiling
namespace {
struct ProfRec {
  const char *name;
  int device;
  cudaEvent_t a, b;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;
std::vector<std::pair<int, cudaEvent_t>> g_event_pool;

cudaEvent_t take_event(int dev) {
  for (size_t i = 0; i < g_event_pool.size(); i++)
    if (g_event_pool[i].first == dev) {
      cudaEvent_t e = g_event_pool[i].second;
      g_event_pool.erase(g_event_pool.begin() + i);
      return e;
    }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

bool profiling_enabled() { return g_prof_on; }

bool nvtx_enabled() {
  static const bool on = [] {
    const char *v = getenv("ZKB_NVTX");
    return v && *v && *v != '0';
  }();
  return on;
}
void nvtx_push(const char *name) { nvtxRangePushA(name); }
void nvtx_pop() { nvtxRangePop(); }

int prof_record(const char *name, cudaStream_t s, int phase, void **token) {
  if (phase == 0) {
    // launches recorded into a CUDA graph are not timed one by one
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      return ZKB_OK;
    }
  }
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (phase == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    ProfRec r{name, dev, take_event(dev), take_event(dev)};
    cudaEventRecord(r.a, s);
    g_prof.push_back(r);
    *token = (void *)(uintptr_t)g_prof.size();  // 1-based index
  } else {
    size_t idx = (size_t)(uintptr_t)*token - 1;
    if (idx < g_prof.size()) cudaEventRecord(g_prof[idx].b, s);
    *token = nullptr;
  }
  return ZKB_OK;
}

int profile_start() {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto &r : g_prof) {
    g_event_pool.push_back({r.device, r.a});
    g_event_pool.push_back({r.device, r.b});
  }
  g_prof.clear();
  g_prof_on = true;
  return ZKB_OK;
}

int profile_stop(zkb_kernel_stat *out, int cap) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = false;
  std::vector<zkb_kernel_stat> agg;
  int prev = 0;
  cudaGetDevice(&prev);
  for (auto &r : g_prof) {
    cudaSetDevice(r.device);
    float ms = 0;
    if (cudaEventSynchronize(r.b) != cudaSuccess || cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) {
      cudaSetDevice(prev);
      set_error("profiling events could not be read");
      return ZKB_ERR_CUDA;
    }
    zkb_kernel_stat *st = nullptr;
    for (auto &a : agg)
      if (strncmp(a.name, r.name, sizeof a.name) == 0) st = &a;
    if (!st) {
      agg.push_back(zkb_kernel_stat{});
      st = &agg.back();
      strncpy(st->name, r.name, sizeof st->name - 1);
    }
    st->launches++;
    st->total_ms += ms;
    st->max_ms = ms > st->max_ms ? ms : st->max_ms;
  }
  cudaSetDevice(prev);
  int n = (int)agg.size();
  for (int i = 0; i < n && i < cap; i++) out[i] = agg[i];
  return n;
}

// ------------------------------------------------------- failure detection
// The reference's watchdog and circuit breaker (zkf-metal/src/async_dispatch.rs:16-71,
// 162-204; device.rs:649-662): every host wait on device work has a deadline, and a
// device error or an expired deadline opens a process-wide circuit after which the
// entry points decline (the caller takes its CPU path) until it is reset.
namespace {
std::atomic<bool> g_circuit{false};
std::mutex g_circuit_mu;
std::string g_circuit_why;
std::atomic<int> g_inject_oom{0}, g_inject_timeout{0};

long watchdog_ms() {
  static const long ms = [] {
    const char *v = getenv("ZKB_WATCHDOG_MS");
    return v && *v ? strtol(v, nullptr, 10) : 120000L;
  }();
  return ms;
}

bool take_injected(std::atomic<int> &counter) {
  int c = counter.load();
  while (c > 0)
    if (counter.compare_exchange_weak(c, c - 1)) return true;
  return false;
}
}  // namespace

bool library_disabled() {
  static const bool off = [] {
    const char *v = getenv("ZKB_DISABLE");
    return v && *v && *v != '0';
  }();
  return off;
}

void trip_circuit(const char *why) {
  std::lock_guard<std::mutex> lk(g_circuit_mu);
  if (!g_circuit.load()) g_circuit_why = why;
  g_circuit.store(true);
}

bool circuit_open(std::string *why) {
  if (!g_circuit.load()) return false;
  if (why) {
    std::lock_guard<std::mutex> lk(g_circuit_mu);
    *why = g_circuit_why;
  }
  return true;
}

int library_gate() {
  if (library_disabled()) {
    set_error("disabled by ZKB_DISABLE");
    return ZKB_DECLINED;
  }
  std::string why;
  if (circuit_open(&why)) {
    set_error("circuit open after a device failure (%s); zkb_circuit_reset() closes it", why.c_str());
    return ZKB_DECLINED;
  }
  return ZKB_OK;
}

void circuit_reset() {
  std::lock_guard<std::mutex> lk(g_circuit_mu);
  g_circuit.store(false);
  g_circuit_why.clear();
}

int inject_fault(int kind, int count) {
  if (count < 0) return ZKB_ERR_INVALID;
  if (kind == 1)
    g_inject_oom.store(count);
  else if (kind == 2)
    g_inject_timeout.store(count);
  else
    return ZKB_ERR_INVALID;
  return ZKB_OK;
}

int wait_stream(cudaStream_t s) {
  if (take_injected(g_inject_timeout)) {
    // simulated expiry: the work is let finish first, so nothing stays in flight
    cudaStreamSynchronize(s);
    trip_circuit("watchdog: a stream wait exceeded its deadline (injected)");
    set_error("watchdog: stream wait exceeded %ld ms (injected)", watchdog_ms());
    return ZKB_ERR_TIMEOUT;
  }
  const long ms = watchdog_ms();
  cudaError_t e;
  if (ms <= 0) {
    e = cudaStreamSynchronize(s);
  } else {
    using clk = std::chrono::steady_clock;
    const auto deadline = clk::now() + std::chrono::milliseconds(ms);
    int polls = 0;
    for (;;) {
      e = cudaStreamQuery(s);
      if (e != cudaErrorNotReady) break;
      if (clk::now() > deadline) {
        trip_circuit("watchdog: a stream wait exceeded its deadline");
        set_error("watchdog: stream wait exceeded %ld ms", ms);
        return ZKB_ERR_TIMEOUT;
      }
      // spin briefly for short waits, then back off to a few tens of microseconds
      if (++polls < 64)
        std::this_thread::yield();
      else
        std::this_thread::sleep_for(std::chrono::microseconds(polls < 256 ? 5 : 20));
    }
  }
  if (e != cudaSuccess) {
    trip_circuit(cudaGetErrorString(e));
    set_error("device work failed: %s", cudaGetErrorString(e));
    return ZKB_ERR_CUDA;
  }
  return ZKB_OK;
}

// Minimum sizes below which the host-pointer entry points and the runtime nodes decline so the caller runs its
// CPU path: the reference's ThresholdConfig (zkf-metal/src/tuning.rs:84-111; ntt = rows,
// poseidon2 = permutations, merkle = leaves, fri = fold outputs), with a runtime override
// (tuning.rs:284-300).  Default: no minimum; env ZKB_THRESHOLDS="ntt=4096,poseidon2=1000,..."
// or zkb_set_thresholds() sets them.
namespace {
std::mutex g_thr_mu;
bool g_thr_init = false;
zkb_thresholds g_thr{};
}  // namespace

zkb_thresholds thresholds() {
  std::lock_guard<std::mutex> lk(g_thr_mu);
  if (!g_thr_init) {
    g_thr_init = true;
    if (const char *v = getenv("ZKB_THRESHOLDS")) {
      std::string spec(v);
      size_t pos = 0;
      while (pos < spec.size()) {
        size_t end = spec.find(',', pos);
        if (end == std::string::npos) end = spec.size();
        const std::string kv = spec.substr(pos, end - pos);
        const size_t eq = kv.find('=');
        if (eq != std::string::npos) {
          const std::string k = kv.substr(0, eq);
          const uint64_t x = strtoull(kv.c_str() + eq + 1, nullptr, 10);
          if (k == "ntt") g_thr.ntt = x;
          else if (k == "poseidon2") g_thr.poseidon2 = x;
          else if (k == "merkle") g_thr.merkle = x;
          else if (k == "fri") g_thr.fri = x;
        }
        pos = end + 1;
      }
    }
  }
  return g_thr;
}

int below(uint64_t size, uint64_t minimum, const char *what) {
  if (size < minimum) {
    set_error("below threshold: %s size %llu < %llu (use the CPU path)", what, (unsigned long long)size,
              (unsigned long long)minimum);
    return ZKB_DECLINED;
  }
  return ZKB_OK;
}

void set_thresholds(const zkb_thresholds &t) {
  thresholds();  // the environment is read before an override replaces it
  std::lock_guard<std::mutex> lk(g_thr_mu);
  g_thr = t;
}

namespace {
std::atomic<uint64_t> g_device_allocs{0};
std::atomic<uint64_t> g_pool_allocs{0};
}

void note_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }
uint64_t device_alloc_count() { return g_device_allocs.load(std::memory_order_relaxed); }
uint64_t pool_alloc_count() { return g_pool_allocs.load(std::memory_order_relaxed); }

// ---- large blocks: an exact-size cache in front of the stream-ordered pool
// Repeated jobs of one shape ask for the same sizes (staged trace, LDE, tree layers, FRI
// state).  A freed block of at least kCacheMin bytes is kept, with an event recorded on the
// stream that freed it, and the next request of the same rounded size on the same device
// takes it: on the stream that freed it at once (stream order), on any other stream once
// that event has completed — no dependency on another stream's queued work is inserted.  Without the cache, pool fragmentation made the pool grow (map and
// clear fresh memory) in the middle of jobs, stalls of hundreds of milliseconds.  When the
// pool runs out of memory the cached blocks go back to it and the request is retried.
// Allocations and frees on a capturing stream bypass the cache (graph memory nodes).
namespace {
constexpr size_t kCacheMin = 1u << 20;
constexpr size_t kCacheRound = 2u << 20;
struct CachedBlock {
  void *p;
  cudaEvent_t freed;
  cudaStream_t stream;  // the stream that freed it
};
std::mutex g_cache_mu;
std::map<void *, std::pair<size_t, int>> g_cache_live;            // block -> (rounded size, device)
std::multimap<std::pair<int, size_t>, CachedBlock> g_cache_free;   // (device, size) -> blocks

bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// Returns the cached blocks of `dev` to the pool (on s, after their frees); with
// `completed_only`, only those whose free has completed.  Called with g_cache_mu held.
void cache_flush(int dev, cudaStream_t s, bool completed_only) {
  for (auto it = g_cache_free.begin(); it != g_cache_free.end();) {
    if (it->first.first != dev || (completed_only && cudaEventQuery(it->second.freed) != cudaSuccess)) {
      ++it;
      continue;
    }
    cudaStreamWaitEvent(s, it->second.freed, 0);
    cudaFreeAsync(it->second.p, s);
    cudaEventDestroy(it->second.freed);
    it = g_cache_free.erase(it);
  }
}
}  // namespace

int dev_alloc(void **p, size_t bytes, cudaStream_t s) {
  note_device_alloc();
  if (take_injected(g_inject_oom)) {
    *p = nullptr;
    set_error("device allocation of %zu bytes failed: out of memory (injected)", bytes);
    return ZKB_ERR_OOM;
  }
  const bool cached = bytes >= kCacheMin && !capturing(s);
  const size_t rb = cached ? (bytes + kCacheRound - 1) / kCacheRound * kCacheRound : bytes;
  int dev = 0;
  if (cached) {
    ZKB_CHECK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_cache_mu);
    // a block freed on this stream is ordered before this use by the stream itself (the
    // wait on its event costs nothing and stays correct if the handle was recycled); one
    // freed on another stream only once its free has completed
    auto range = g_cache_free.equal_range({dev, rb});
    auto pick = range.second;
    for (auto it = range.first; it != range.second; ++it) {
      if (it->second.stream == s) {
        pick = it;
        break;
      }
      if (pick == range.second && cudaEventQuery(it->second.freed) == cudaSuccess) pick = it;
    }
    if (pick != range.second) {
      *p = pick->second.p;
      if (pick->second.stream == s) cudaStreamWaitEvent(s, pick->second.freed, 0);
      cudaEventDestroy(pick->second.freed);
      g_cache_free.erase(pick);
      g_cache_live[*p] = {rb, dev};
      return ZKB_OK;
    }
  }
  if (cached) g_pool_allocs.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaMallocAsync(p, rb, s);
  if (e == cudaErrorMemoryAllocation && cached) {
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(g_cache_mu);
    cache_flush(dev, s, true);
    e = cudaMallocAsync(p, rb, s);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      cache_flush(dev, s, false);
      e = cudaMallocAsync(p, rb, s);
    }
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? ZKB_ERR_OOM : ZKB_ERR_CUDA;
  }
  if (cached) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_cache_live[*p] = {rb, dev};
  }
  return ZKB_OK;
}

int release_cached_memory() {
  int dev = 0;
  ZKB_CHECK_CUDA(cudaGetDevice(&dev));
  cudaStream_t s = nullptr;
  ZKB_CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    cache_flush(dev, s, false);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  ZKB_CHECK_CUDA(e);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) ZKB_CHECK_CUDA(cudaMemPoolTrimTo(pool, 0));
  return ZKB_OK;
}

void dev_free(void *p, cudaStream_t s) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache_live.find(p);
    if (it != g_cache_live.end()) {
      const std::pair<int, size_t> key{it->second.second, it->second.first};
      g_cache_live.erase(it);
      cudaEvent_t ev = nullptr;
      if (!capturing(s) && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
        if (cudaEventRecord(ev, s) == cudaSuccess) {
          g_cache_free.insert({key, CachedBlock{p, ev, s}});
          return;
        }
        cudaEventDestroy(ev);
      }
    }
  }
  cudaFreeAsync(p, s);
}

}  // namespace zkb
