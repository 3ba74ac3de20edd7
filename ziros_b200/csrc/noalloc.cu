// noalloc.cu — a column DFT that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a prover embedded in a process whose device
// memory is owned by another allocator (a framework that reserves the whole GPU when
// it starts leaves nothing for a side allocation), or a latency-critical loop that
// must not pay the device-wide synchronisation an allocation or a free can cause.
// zkb_dft_batch_noalloc_dev serves them: its scratch — the twiddle table and the
// out-of-place buffer of the transform — is the fixed array below, which every GPU
// that loads this library holds until the process exits.
//
// The array is shared by every call on a device and keeps the contents of the last
// call.  Nothing in it has to start at zero: each call regenerates the twiddle table
// and overwrites the whole temp region before reading it.  Calls whose work overlaps on
// the GPU (different streams, or different host threads) race on the array; issue them
// on one stream or serialise them.
#include <mutex>

#include "common.cuh"
#include "engine.cuh"

namespace zkb {

// Upper bound of the scratch: twiddle table (2^log_h elements, padded to 256 bytes)
// plus the temp copy of the matrix (2^log_h x width elements).
constexpr size_t kNoAllocScratchBytes = 16u << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_scratch_mu;
struct ScratchSlot {
  void *ctx = nullptr;  // CUcontext the address belongs to
  void *ptr = nullptr;
};
ScratchSlot g_scratch_dev[64];

// cuCtxGetCurrent, fetched from the driver at run time (the library does not link
// libcuda, so it still loads on a machine without a driver).
using CtxGetCurrentFn = int (*)(void **);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (CtxGetCurrentFn) nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

void *current_ctx() {
  void *c = nullptr;
  CtxGetCurrentFn fn = ctx_get_current();
  if (!fn || fn(&c) != 0) return nullptr;
  return c;
}

// The symbol's name is a host-side stand-in, not a device address.  Set-up, once per
// device with that device current (the first call on the device): cudaGetSymbolAddress
// gives the array's address in the device's context.  The address is kept with the
// context it belongs to; if the context was torn down and re-created (cudaDeviceReset),
// the module was reloaded elsewhere and the lookup runs again.
int scratch_address(void **out) {
  int dev = 0;
  ZKB_CHECK_CUDA(cudaGetDevice(&dev));
  ZKB_REQUIRE(dev >= 0 && dev < 64, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  ScratchSlot &slot = g_scratch_dev[dev];
  void *ctx = current_ctx();
  if (!slot.ptr || ctx == nullptr || ctx != slot.ctx) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("cudaGetSymbolAddress of the allocation-free scratch failed: %s", cudaGetErrorString(e));
      return ZKB_ERR_CUDA;
    }
    slot.ptr = p;
    slot.ctx = current_ctx();  // the lookup made the device's primary context current
  }
  *out = slot.ptr;
  return ZKB_OK;
}

template <class F>
int dft_noalloc(void *d, uint32_t log_h, uint32_t width, int inverse, cudaStream_t s) {
  using T = typename F::T;
  ZKB_REQUIRE(log_h <= (uint32_t)F::TWO_ADICITY, "log_h %u exceeds the two-adicity", log_h);
  const uint64_t n = 1ull << log_h;
  const uint64_t tw_bytes = ((n * sizeof(T)) + 255) & ~255ull;
  const uint64_t need = tw_bytes + n * (uint64_t)width * sizeof(T);
  if (need > kNoAllocScratchBytes) {
    set_error("zkb_dft_batch_noalloc_dev: 2^%u x %u matrix needs %llu scratch bytes, more than the "
              "%zu-byte fixed scratch; use zkb_dft_batch_dev",
              log_h, width, (unsigned long long)need, kNoAllocScratchBytes);
    return ZKB_ERR_INVALID;
  }
  void *base = nullptr;
  ZKB_TRY(scratch_address(&base));
  T *tw = static_cast<T *>(base);
  T *tmp = reinterpret_cast<T *>(static_cast<unsigned char *>(base) + tw_bytes);
  return ntt_dft_into<F>(static_cast<T *>(d), (int)log_h, width, inverse != 0, tw, tmp, s);
}
}  // namespace

}  // namespace zkb

extern "C" int zkb_dft_batch_noalloc_dev(int field, void *d_rowmajor, uint32_t log_h, uint32_t width,
                                         int inverse, void *stream) {
  using namespace zkb;
  clear_error();
  ZKB_TRY(library_gate());  // kill switch and open circuit decline, as in every entry point
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    set_error("no CUDA device available");
    return ZKB_DECLINED;
  }
  ZKB_REQUIRE(field == ZKB_FIELD_BABYBEAR || field == ZKB_FIELD_GOLDILOCKS, "unknown field %d", field);
  ZKB_REQUIRE(d_rowmajor != nullptr || width == 0, "null matrix");
  cudaStream_t s = (cudaStream_t)stream;
  if (field == ZKB_FIELD_BABYBEAR) return dft_noalloc<BabyBear>(d_rowmajor, log_h, width, inverse, s);
  return dft_noalloc<Goldilocks>(d_rowmajor, log_h, width, inverse, s);
}
