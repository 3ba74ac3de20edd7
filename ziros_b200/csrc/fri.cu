// fri.cu — FRI folding by 2 (base field and the BabyBear quartic extension).
//
// Base field: FriAccelerator::fold_* / MetalFri (zkf-core/src/acceleration.rs:197-217,
// zkf-metal/src/shaders/fri.metal:14-53):
//   out[i] = (e[2i] + e[2i+1]) / 2 + alpha * (e[2i] - e[2i+1]) * inv_tw[i].
// Extension: p3 TwoAdicFriFolding::fold_matrix with arity 2 over
// BinomialExtensionField<BabyBear, 4> (x^4 = 11):
//   out[i] = (r0 + r1)/2 + (beta/2) * g^-rev(i) * (r0 - r1),  g = w_{2 n_out},
// the rows (r0, r1) being the values at +x and -x of the bit-reversed domain.
#include "common.cuh"
#include "engine.cuh"
#include "field.cuh"

namespace zkb {

// canonical x canonical -> canonical
template <class F>
__device__ __forceinline__ typename F::T mul_cc(typename F::T a, typename F::T b);
template <>
__device__ __forceinline__ uint32_t mul_cc<BabyBear>(uint32_t a, uint32_t b) {
  return BabyBear::mont(BabyBear::mont(a, b), BabyBear::R2);
}
template <>
__device__ __forceinline__ uint64_t mul_cc<Goldilocks>(uint64_t a, uint64_t b) {
  return Goldilocks::mul(a, b);
}

// inv_tw given (canonical): the reference formula verbatim.
template <class F>
__global__ void fri_fold_given_kernel(const typename F::T *__restrict__ e, typename F::T *__restrict__ out,
                                      uint64_t n_out, typename F::T alpha_enc,
                                      typename F::T inv2_enc,
                                      const typename F::T *__restrict__ inv_tw) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x) {
    typename F::T a = e[2 * i], b = e[2 * i + 1];
    typename F::T sum = F::mul_tw(F::add(a, b), inv2_enc);
    typename F::T d = F::mul_tw(mul_cc<F>(F::sub(a, b), inv_tw[i]), alpha_enc);
    out[i] = F::add(sum, d);
  }
}

// inv_tw computed: inv_tw[i] = g^-rev(i) / 2 from the cached inverse table of size 2*n_out.
template <class F>
__global__ void fri_fold_p3_kernel(const typename F::T *__restrict__ e, typename F::T *__restrict__ out,
                                   uint64_t n_out, int log_n, typename F::T alpha_enc,
                                   typename F::T inv2_enc,
                                   const typename F::T *__restrict__ itw) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x) {
    typename F::T a = e[2 * i], b = e[2 * i + 1];
    uint64_t r = log_n ? (__brevll(i) >> (64 - log_n)) : 0;
    typename F::T d = F::mul_tw(F::mul_tw(F::sub(a, b), itw[r]), alpha_enc);
    out[i] = F::mul_tw(F::add(F::add(a, b), d), inv2_enc);
  }
}

template <class F>
int fri_fold_base_dev(const typename F::T *d_evals, size_t n_out, typename F::T alpha,
                      const typename F::T *d_inv_tw, typename F::T *d_out, cudaStream_t s) {
  using T = typename F::T;
  if (n_out == 0) return ZKB_OK;
  ZKB_REQUIRE(alpha < F::P, "alpha is not a canonical field element");
  const T inv2 = Dom<F>::encode(inv_host<F>(2));
  const T a_enc = Dom<F>::encode(alpha);
  if (d_inv_tw) {
    ZKB_LAUNCH("fri_fold", s, fri_fold_given_kernel<F><<<grid_for(n_out, 256), 256, 0, s>>>(d_evals, d_out, n_out, a_enc, inv2,
                                                                  d_inv_tw));
  } else {
    int log_n = ilog2_exact(n_out);
    ZKB_REQUIRE(log_n >= 0, "n_out must be a power of two when inv_twiddles is NULL");
    const T *itw;
    ZKB_TRY(get_twiddles<F>(log_n + 1, true, &itw, s));
    ZKB_LAUNCH("fri_fold", s, fri_fold_p3_kernel<F><<<grid_for(n_out, 256), 256, 0, s>>>(d_evals, d_out, n_out, log_n, a_enc,
                                                               inv2, itw));
  }
  ZKB_CHECK_LAUNCH();
  return ZKB_OK;
}

// ---------------------------------------------------------- quartic extension
struct Ext4 {
  uint32_t c[4];
};

// a * b with b encoded (Montgomery) coefficientwise; x^4 = 11.
__device__ __forceinline__ Ext4 ext4_mul_enc(const Ext4 &a, const Ext4 &b_enc) {
  using B = BabyBear;
  uint32_t p[7];
#pragma unroll
  for (int k = 0; k < 7; k++) p[k] = 0;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) p[i + j] = B::add(p[i + j], B::mont(a.c[i], b_enc.c[j]));
  Ext4 r;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint32_t h = p[k + 4];
    const uint32_t h2 = B::add(h, h), h4 = B::add(h2, h2), h8 = B::add(h4, h4);
    r.c[k] = B::add(p[k], B::add(B::add(h8, h2), h));  // + 11 h
  }
  r.c[3] = p[3];
  return r;
}

struct Ext4Params {
  Ext4 half_beta_enc;  // beta / 2, Montgomery-encoded coefficients
  uint32_t inv2_enc;
};

__global__ void fri_fold_ext4_kernel(const uint32_t *__restrict__ e, uint32_t *__restrict__ out,
                                     uint64_t n_out, int log_n, const Ext4Params prm,
                                     const uint32_t *__restrict__ itw) {
  using B = BabyBear;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 r0 = reinterpret_cast<const uint4 *>(e)[2 * i];
    const uint4 r1 = reinterpret_cast<const uint4 *>(e)[2 * i + 1];
    uint64_t r = log_n ? (__brevll(i) >> (64 - log_n)) : 0;
    const uint32_t w = itw[r];
    Ext4 d;
    d.c[0] = B::mul_tw(B::sub(r0.x, r1.x), w);
    d.c[1] = B::mul_tw(B::sub(r0.y, r1.y), w);
    d.c[2] = B::mul_tw(B::sub(r0.z, r1.z), w);
    d.c[3] = B::mul_tw(B::sub(r0.w, r1.w), w);
    Ext4 t = ext4_mul_enc(d, prm.half_beta_enc);
    uint4 o;
    o.x = B::add(B::mul_tw(B::add(r0.x, r1.x), prm.inv2_enc), t.c[0]);
    o.y = B::add(B::mul_tw(B::add(r0.y, r1.y), prm.inv2_enc), t.c[1]);
    o.z = B::add(B::mul_tw(B::add(r0.z, r1.z), prm.inv2_enc), t.c[2]);
    o.w = B::add(B::mul_tw(B::add(r0.w, r1.w), prm.inv2_enc), t.c[3]);
    reinterpret_cast<uint4 *>(out)[i] = o;
  }
}

int fri_fold_ext4_dev(const uint32_t *d_evals, size_t n_out, const uint32_t beta[4],
                      uint32_t *d_out, cudaStream_t s) {
  if (n_out == 0) return ZKB_OK;
  int log_n = ilog2_exact(n_out);
  ZKB_REQUIRE(log_n >= 0, "n_out must be a power of two");
  ZKB_REQUIRE(((uintptr_t)d_evals & 15) == 0 && ((uintptr_t)d_out & 15) == 0,
              "extension buffers must be 16-byte aligned");
  Ext4Params prm;
  const uint32_t inv2 = inv_host<BabyBear>(2);
  for (int k = 0; k < 4; k++) {
    ZKB_REQUIRE(beta[k] < BabyBear::P, "beta is not canonical");
    prm.half_beta_enc.c[k] = BabyBear::tw_encode(BabyBear::mul_host(beta[k], inv2));
  }
  prm.inv2_enc = BabyBear::tw_encode(inv2);
  const uint32_t *itw;
  ZKB_TRY(get_twiddles<BabyBear>(log_n + 1, true, &itw, s));
  ZKB_LAUNCH("fri_fold_ext4", s, fri_fold_ext4_kernel<<<grid_for(n_out, 256), 256, 0, s>>>(d_evals, d_out, n_out, log_n, prm, itw));
  ZKB_CHECK_LAUNCH();
  return ZKB_OK;
}

template int fri_fold_base_dev<BabyBear>(const uint32_t *, size_t, uint32_t, const uint32_t *,
                                         uint32_t *, cudaStream_t);
template int fri_fold_base_dev<Goldilocks>(const uint64_t *, size_t, uint64_t, const uint64_t *,
                                           uint64_t *, cudaStream_t);

}  // namespace zkb
