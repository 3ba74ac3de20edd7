// poly.cu — polynomial operations of the reference's PolyOpsAccelerator
// (zkf-core/src/acceleration.rs:173-194; Metal implementation zkf-metal/src/poly.rs:37-230):
//   batch evaluation   f(x_j) = sum_i c_i x_j^i by Horner, one point per thread;
//   coset evaluation   f(shift * w^i), i < 2^log_n: coefficients times shift^i, then the
//                      natural-order DFT (poly.rs:160-190);
//   quotient           (e_i - f(z)) / (x_i - z) with x_i = w^i on the canonical subgroup of
//                      size 2^log_n, 0 where x_i = z (poly.rs:192-230 and its test :366-400).
// The quotient inverts its denominators in runs of QB per thread (Montgomery's trick:
// one field inversion per run, three products per element).
#include "common.cuh"
#include "engine.cuh"

namespace zkb {
namespace {

using GL = Goldilocks;

__device__ __forceinline__ uint64_t gl_pow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = GL::mul(r, a);
    a = GL::mul(a, a);
    e >>= 1;
  }
  return r;
}

__global__ void poly_eval_kernel(const uint64_t *__restrict__ coeffs, uint64_t n_coeffs,
                                 const uint64_t *__restrict__ pts, uint64_t n_pts, uint64_t *__restrict__ out) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_pts;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = pts[j];
    uint64_t r = 0;
    for (uint64_t i = n_coeffs; i-- > 0;) r = GL::add(GL::mul(r, x), coeffs[i]);
    out[j] = r;
  }
}

// c_i <- c_i * shift^i: each thread starts from shift^(first index) and steps by shift
__global__ void shift_powers_kernel(uint64_t *__restrict__ c, uint64_t n, uint64_t shift, uint32_t per_thread) {
  const uint64_t i0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * per_thread;
  if (i0 >= n) return;
  uint64_t p = gl_pow(shift, i0);
  for (uint32_t k = 0; k < per_thread && i0 + k < n; k++) {
    c[i0 + k] = GL::mul(c[i0 + k], p);
    p = GL::mul(p, shift);
  }
}

constexpr int QB = 16;

__global__ void quotient_kernel(const uint64_t *__restrict__ e, uint64_t n, uint64_t w, uint64_t z, uint64_t fz,
                                uint64_t *__restrict__ out) {
  const uint64_t i0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * QB;
  if (i0 >= n) return;
  const int m = (int)(n - i0 < (uint64_t)QB ? n - i0 : QB);
  uint64_t d[QB], prefix[QB];
  uint64_t x = gl_pow(w, i0), acc = 1;
#pragma unroll
  for (int k = 0; k < QB; k++) {
    if (k < m) {
      d[k] = GL::sub(x, z);
      prefix[k] = acc;
      if (d[k] != 0) acc = GL::mul(acc, d[k]);  // a vanishing denominator is left out of the product
      x = GL::mul(x, w);
    }
  }
  uint64_t inv = gl_pow(acc, GL::P - 2);  // inverse of the product of the nonzero denominators
#pragma unroll
  for (int k = QB - 1; k >= 0; k--) {
    if (k < m) {
      if (d[k] == 0) {
        out[i0 + k] = 0;
      } else {
        const uint64_t inv_d = GL::mul(inv, prefix[k]);
        inv = GL::mul(inv, d[k]);
        out[i0 + k] = GL::mul(GL::sub(e[i0 + k], fz), inv_d);
      }
    }
  }
}

int upload(ScratchBuf &b, const void *h, size_t bytes, cudaStream_t s) {
  ZKB_TRY(b.alloc(bytes ? bytes : 8, s));
  if (bytes) ZKB_CHECK_CUDA(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, s));
  return ZKB_OK;
}

int download(void *h, const ScratchBuf &b, size_t bytes, cudaStream_t s) {
  if (bytes) ZKB_CHECK_CUDA(cudaMemcpyAsync(h, b.p, bytes, cudaMemcpyDeviceToHost, s));
  return wait_stream(s);
}

int check_canonical(const uint64_t *v, size_t n, const char *what) {
  for (size_t i = 0; i < n; i++) ZKB_REQUIRE(v[i] < GL::P, "%s[%zu] is not canonical", what, i);
  return ZKB_OK;
}

}  // namespace
}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_poly_eval_goldilocks(const uint64_t *coeffs, size_t n_coeffs, const uint64_t *points, size_t n_points,
                             uint64_t *out) {
  clear_error();
  ZKB_TRY(library_gate());
  ZKB_REQUIRE((coeffs || !n_coeffs) && (points || !n_points) && (out || !n_points), "null buffers");
  ZKB_TRY(check_canonical(coeffs, n_coeffs, "coeffs"));
  ZKB_TRY(check_canonical(points, n_points, "points"));
  if (n_points == 0) return ZKB_OK;
  cudaStream_t s = thread_stream();
  ScratchBuf dc, dp, dout;
  ZKB_TRY(upload(dc, coeffs, n_coeffs * 8, s));
  ZKB_TRY(upload(dp, points, n_points * 8, s));
  ZKB_TRY(dout.alloc(n_points * 8, s));
  ZKB_LAUNCH("poly_eval", s, poly_eval_kernel<<<grid_for(n_points, 256), 256, 0, s>>>(dc.as<uint64_t>(), n_coeffs, dp.as<uint64_t>(), n_points, dout.as<uint64_t>()));
  return download(out, dout, n_points * 8, s);
}

int zkb_poly_coset_eval_goldilocks(const uint64_t *coeffs, uint32_t log_n, uint64_t shift, uint64_t *out) {
  clear_error();
  ZKB_TRY(library_gate());
  ZKB_REQUIRE(coeffs && out && log_n <= 30, "bad arguments");
  ZKB_REQUIRE(shift < GL::P, "shift is not canonical");
  const uint64_t n = 1ull << log_n;
  ZKB_TRY(check_canonical(coeffs, n, "coeffs"));
  cudaStream_t s = thread_stream();
  ScratchBuf d;
  ZKB_TRY(upload(d, coeffs, n * 8, s));
  const uint32_t per = 64;
  ZKB_LAUNCH("poly_coset_shift", s, shift_powers_kernel<<<(unsigned)((n + 256ull * per - 1) / (256ull * per)), 256, 0, s>>>(d.as<uint64_t>(), n, shift, per));
  ZKB_TRY(ntt_dft_dev<Goldilocks>(d.as<uint64_t>(), (int)log_n, 1, false, s));
  return download(out, d, n * 8, s);
}

int zkb_poly_quotient_goldilocks(const uint64_t *evals, uint32_t log_n, uint64_t z, uint64_t f_z, uint64_t *out) {
  clear_error();
  ZKB_TRY(library_gate());
  ZKB_REQUIRE(evals && out && log_n <= 32, "bad arguments");
  ZKB_REQUIRE(z < GL::P && f_z < GL::P, "z or f(z) is not canonical");
  const uint64_t n = 1ull << log_n;
  ZKB_TRY(check_canonical(evals, n, "evals"));
  cudaStream_t s = thread_stream();
  ScratchBuf de, dout;
  ZKB_TRY(upload(de, evals, n * 8, s));
  ZKB_TRY(dout.alloc(n * 8, s));
  const uint64_t w = two_adic_generator<Goldilocks>((int)log_n);
  const uint64_t threads = (n + QB - 1) / QB;
  ZKB_LAUNCH("poly_quotient", s, quotient_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(de.as<uint64_t>(), n, w, z, f_z, dout.as<uint64_t>()));
  return download(out, dout, n * 8, s);
}

}  // extern "C"
