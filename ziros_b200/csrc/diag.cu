// diag.cu — measured integer-multiply ceiling used as the Poseidon2 roofline peak.
//
// Every thread runs 8 independent chains of field multiplications (the same
// Montgomery / Goldilocks multiply the kernels use) on all SMs; the result is
// field multiplications per second.  A Poseidon2 kernel's achieved rate of
// algorithmic field multiplications divided by this figure is the fraction of the
// multiply throughput it sustains once its additions and data movement are paid.
#include "common.cuh"
#include "field.cuh"

namespace zkb {

template <class F>
__global__ void __launch_bounds__(256) mul_chain_kernel(typename F::T *sink, int iters,
                                                        typename F::T k) {
  using T = typename F::T;
  T a[8];
#pragma unroll
  for (int j = 0; j < 8; j++) a[j] = (T)(threadIdx.x * 8 + j + 1 + blockIdx.x);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = Dom<F>::mul(a[j], k);
  }
  T acc = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) acc ^= a[j];
  if (acc == (T)0x12345) sink[0] = acc;  // keeps the chains live
}

template <class F>
static int mul_peak(double *mul_per_s) {
  using T = typename F::T;
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));
  cudaStream_t s = thread_stream();
  ScratchBuf sink;
  ZKB_TRY(sink.alloc(sizeof(T), s));
  const int blocks = ctx->sm_count * 8, threads = 256, iters = sizeof(T) == 4 ? 4096 : 1024;
  cudaEvent_t a, b;
  ZKB_CHECK_CUDA(cudaEventCreate(&a));
  ZKB_CHECK_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(a, s);
    mul_chain_kernel<F><<<blocks, threads, 0, s>>>(sink.as<T>(), iters, (T)0x1234567);
    cudaEventRecord(b, s);
    ZKB_CHECK_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0 && ms < best) best = ms;  // first launch is a warm-up
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  ZKB_CHECK_LAUNCH();
  *mul_per_s = (double)blocks * threads * iters * 8 / (best * 1e-3);
  return ZKB_OK;
}

int measure_mul_peak(int field, double *mul_per_s) {
  if (field == ZKB_FIELD_BABYBEAR) return mul_peak<BabyBear>(mul_per_s);
  return mul_peak<Goldilocks>(mul_per_s);
}

}  // namespace zkb
