// common.cuh — status codes, last-error convention, device context and memory.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "../../include/zkb200.h"

namespace zkb {

// Sets the thread-local last-error message (zkf-ffi set_last_error, zkf-ffi/src/lib.rs:49-60).
void set_error(const char *fmt, ...);
void clear_error();

#define ZKB_CHECK_CUDA(call)                                                          \
  do {                                                                                \
    cudaError_t zkb_e_ = (call);                                                      \
    if (zkb_e_ != cudaSuccess) {                                                      \
      ::zkb::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(zkb_e_),     \
                       __FILE__, __LINE__);                                           \
      return zkb_e_ == cudaErrorMemoryAllocation ? ZKB_ERR_OOM : ZKB_ERR_CUDA;         \
    }                                                                                 \
  } while (0)

#define ZKB_CHECK_LAUNCH() ZKB_CHECK_CUDA(cudaGetLastError())

#define ZKB_TRY(expr)                 \
  do {                                \
    int zkb_rc_ = (expr);             \
    if (zkb_rc_ != ZKB_OK) return zkb_rc_; \
  } while (0)

#define ZKB_REQUIRE(cond, ...)           \
  do {                                   \
    if (!(cond)) {                       \
      ::zkb::set_error(__VA_ARGS__);     \
      return ZKB_ERR_INVALID;            \
    }                                    \
  } while (0)

// A cached device table (twiddles, coset factors).  Owned by the context.  It is built
// on the stream of the call that first needed it; `ready` is recorded after the build, and
// every later user's stream waits for it, so no host thread waits for a build.
struct DeviceTable {
  void *ptr = nullptr;
  size_t bytes = 0;
  cudaEvent_t ready = nullptr;
  bool complete = false;  // `ready` seen complete: later users need not wait
};

// One per CUDA device: caches shared by every stream on that device.
struct DeviceContext {
  int device = -1;
  int sm_count = 0;
  std::mutex mu;
  std::map<std::tuple<int, int, int>, DeviceTable> twiddles;           // (field, log_n, inverse)
  std::map<std::tuple<int, int, int, uint64_t>, DeviceTable> cosets;   // (field, log_n, log_b, shift)
  // coset factors and forward twists in the order the fused LDE kernel reads them
  std::map<std::tuple<int, int, int, uint64_t, int>, DeviceTable> fused;  // (field, log_n, log_b, shift, K)
};

// Context of the calling thread's current device (initialised on first use).
int current_context(DeviceContext **out);
// Stream of the calling thread on its current device (created on first use).
cudaStream_t thread_stream();
// A user stream argument follows CUDA's convention: NULL is the default stream.
inline cudaStream_t resolve_stream(void *s) { return (cudaStream_t)s; }

// Stream-ordered scratch allocation from the device's memory pool.
int dev_alloc(void **p, size_t bytes, cudaStream_t s);
// Every device allocation the library makes (pool or cudaMalloc) is counted here;
// zkb_debug_device_allocations() reads the count.
void note_device_alloc();
uint64_t device_alloc_count();
// Allocations of cached sizes (1 MiB or more) that missed the block cache and took new
// memory from the stream-ordered pool.
uint64_t pool_alloc_count();
// Returns the cached blocks of the current device to the pool and trims the pool's unused
// memory back to the device (for allocations outside the pool, e.g. a batch plan's arena).
int release_cached_memory();
// Host wait on a stream with the watchdog deadline (ZKB_WATCHDOG_MS, default 120 s, 0 =
// none); a device error or an expired deadline opens the circuit.
int wait_stream(cudaStream_t s);
bool library_disabled();
// ZKB_DECLINED (with the reason) when the library is disabled or the circuit is open.
int library_gate();
void trip_circuit(const char *why);
bool circuit_open(std::string *why);
void circuit_reset();
int inject_fault(int kind, int count);
// Fallback thresholds (zkb_set_thresholds / ZKB_THRESHOLDS) and the check that declines.
zkb_thresholds thresholds();
void set_thresholds(const zkb_thresholds &t);
int below(uint64_t size, uint64_t minimum, const char *what);
void dev_free(void *p, cudaStream_t s);

// RAII holder for stream-ordered scratch.
struct ScratchBuf {
  void *p = nullptr;
  cudaStream_t s = nullptr;
  ScratchBuf() = default;
  ScratchBuf(const ScratchBuf &) = delete;
  ScratchBuf &operator=(const ScratchBuf &) = delete;
  ~ScratchBuf() {
    if (p) dev_free(p, s);
  }
  int alloc(size_t bytes, cudaStream_t stream) {
    s = stream;
    return dev_alloc(&p, bytes ? bytes : 16, stream);
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

// ---- kernel timing (zkb_profile_start / zkb_profile_stop) ----
// When enabled, every launch made through ZKB_LAUNCH records a pair of CUDA events
// on its own stream; zkb_profile_stop aggregates the durations per kernel name.
bool profiling_enabled();
int profile_start();
int profile_stop(zkb_kernel_stat *out, int cap);
int prof_record(const char *name, cudaStream_t s, int phase, void **token);

// ZKB_NVTX=1: every launch is also an NVTX range named for its kernel, for ncu's
// --nvtx filters and other NVTX-aware tools (header-only NVTX v3, no library needed).
bool nvtx_enabled();
void nvtx_push(const char *name);
void nvtx_pop();

struct ProfScope {
  void *tok = nullptr;
  cudaStream_t s;
  bool nvtx = false;
  ProfScope(const char *name, cudaStream_t st) : s(st) {
    if (profiling_enabled()) prof_record(name, s, 0, &tok);
    if (nvtx_enabled()) {
      nvtx = true;
      nvtx_push(name);
    }
  }
  ~ProfScope() {
    if (tok) prof_record(nullptr, s, 1, &tok);
    if (nvtx) nvtx_pop();
  }
};

#define ZKB_LAUNCH(name, stream, ...)              \
  do {                                             \
    ::zkb::ProfScope zkb_ps_((name), (stream));    \
    __VA_ARGS__;                                   \
    ZKB_CHECK_LAUNCH();                            \
  } while (0)

inline size_t field_elem_bytes(int field) { return field == ZKB_FIELD_BABYBEAR ? 4 : 8; }

inline int ilog2_exact(uint64_t x) {
  int l = 0;
  while ((1ull << l) < x) l++;
  return (1ull << l) == x ? l : -1;
}

inline uint64_t ceil_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

inline unsigned grid_for(uint64_t n, unsigned threads, unsigned cap = 148u * 64u) {
  uint64_t g = (n + threads - 1) / threads;
  if (g == 0) g = 1;
  return (unsigned)(g < cap ? g : cap);
}

}  // namespace zkb
