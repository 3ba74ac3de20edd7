// context.cu — per-device context, per-thread streams, last-error, scratch memory.
#include <cstdio>
#include <memory>
#include <vector>

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
    // returning memory to the driver between calls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
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

int dev_alloc(void **p, size_t bytes, cudaStream_t s) {
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? ZKB_ERR_OOM : ZKB_ERR_CUDA;
  }
  return ZKB_OK;
}

void dev_free(void *p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

}  // namespace zkb
