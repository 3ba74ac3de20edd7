// poseidon2.cuh — Poseidon2 permutation on the device, one state per thread.
//
// Structure (zkf-metal/src/shaders/poseidon2.metal:1-154 and :157-264;
// zkf-backends/src/wrapping/poseidon2_goldilocks.rs:117-345):
//   external MDS; R_F/2 full rounds (add rc, x^7 on every lane, external MDS);
//   R_P partial rounds (add rc + x^7 on lane 0, s_i <- d_i*s_i + sum(s));
//   R_F/2 full rounds.
// External MDS = M4 [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]] on each 4-lane chunk,
// then every lane adds the sum of its residue class mod 4.
//
// The state lives in registers in the "internal domain": Montgomery form for
// BabyBear (so x^7 and the diagonal products are single Montgomery products),
// canonical for Goldilocks.  Round constants and the diagonal are passed by value
// as a kernel parameter, so they sit in the constant bank and every lane of a
// warp reads the same word (broadcast), which is the access pattern of a
// permutation that is uniform across threads.
#pragma once
#include <type_traits>

#include "field.cuh"

namespace zkb {

template <class F>
using P2Dom = Dom<F>;

// Largest supported instance: width 16, R_F = 8, R_P = 22.
constexpr int P2_MAX_RC = 8 * 16 + 22;

template <class F, int W>
struct P2Params {
  typename F::T rc[P2_MAX_RC];  // internal-domain constants, flat [initial | internal | terminal]
  typename F::T diag[W];        // internal-domain diagonal
  int rounds_f;
  int rounds_p;
  int out;   // digest elements (8 for W16, 4 for W12)
  int rate;  // sponge rate (8)
  int diag_kind;  // 1: the BabyBear width-16 diagonal V (shift/add form), 0: generic products
};

template <class F>
__host__ __device__ __forceinline__ typename F::T p2_sbox(typename F::T x) {
  using D = P2Dom<F>;
  typename F::T x2 = D::mul(x, x);
  typename F::T x3 = D::mul(x2, x);
  typename F::T x4 = D::mul(x2, x2);
  return D::mul(x4, x3);
}

#ifdef __CUDA_ARCH__
// One out-of-line copy of the Goldilocks S-box (four 64-bit products): inlined sixteen
// times per full round the permutation's loop body outgrows the instruction cache and
// the warps wait on instruction fetch; a call per lane costs a few moves instead.
static __device__ __noinline__ uint64_t p2_sbox_goldilocks_call(uint64_t x) {
  return p2_sbox<Goldilocks>(x);
}
#endif

#ifdef __CUDA_ARCH__
// The partial rounds' sixteen diagonal products, out of line for the same reason.
static __device__ __noinline__ uint64_t p2_mul_goldilocks_call(uint64_t x, uint64_t d) {
  return Goldilocks::mul(x, d);
}
#endif

template <class F>
__host__ __device__ __forceinline__ typename F::T p2_diag_lane(typename F::T x, typename F::T d) {
#ifdef __CUDA_ARCH__
  if constexpr (std::is_same<F, Goldilocks>::value) return p2_mul_goldilocks_call(x, d);
#endif
  return P2Dom<F>::mul(x, d);
}

template <class F>
__host__ __device__ __forceinline__ typename F::T p2_sbox_lane(typename F::T x) {
#ifdef __CUDA_ARCH__
  if constexpr (std::is_same<F, Goldilocks>::value) return p2_sbox_goldilocks_call(x);
#endif
  return p2_sbox<F>(x);
}

template <class F, int W>
__host__ __device__ __forceinline__ void p2_ext_mds(typename F::T (&s)[W]) {
  using D = P2Dom<F>;
  using T = typename F::T;
#pragma unroll
  for (int c = 0; c < W; c += 4) {
    T a = s[c], b = s[c + 1], x = s[c + 2], y = s[c + 3];
    T t01 = D::add(a, b), t23 = D::add(x, y), t0123 = D::add(t01, t23);
    T t01123 = D::add(t0123, b), t01233 = D::add(t0123, y);
    s[c] = D::add(t01123, t01);
    s[c + 1] = D::add(t01123, D::add(x, x));
    s[c + 2] = D::add(t01233, t23);
    s[c + 3] = D::add(t01233, D::add(a, a));
  }
  T sums[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    sums[k] = s[k];
#pragma unroll
    for (int c = 4; c < W; c += 4) sums[k] = D::add(sums[k], s[c + k]);
  }
#pragma unroll
  for (int i = 0; i < W; i++) s[i] = D::add(s[i], sums[i & 3]);
}

template <class F, int W>
__host__ __device__ __forceinline__ void p2_full_round(typename F::T (&s)[W], const typename F::T *rc) {
  using D = P2Dom<F>;
#pragma unroll
  for (int i = 0; i < W; i++) s[i] = p2_sbox_lane<F>(D::add(s[i], rc[i]));
  p2_ext_mds<F, W>(s);
}

template <class F, int W>
__host__ __device__ __forceinline__ void p2_partial_round(typename F::T (&s)[W], typename F::T rc,
                                                 const typename F::T *diag) {
  using D = P2Dom<F>;
  using T = typename F::T;
  s[0] = p2_sbox_lane<F>(D::add(s[0], rc));
  T sum = s[0];
#pragma unroll
  for (int i = 1; i < W; i++) sum = D::add(sum, s[i]);
#pragma unroll
  for (int i = 0; i < W; i++) s[i] = D::add(p2_diag_lane<F>(s[i], diag[i]), sum);
}

// ------------------------------------------------ BabyBear width 16, specialised
// Same permutation, cheaper arithmetic: lazy Montgomery products inside the S-box
// (three corrections instead of four), and the internal diagonal
// V = [-2, 1, 2, 1/2, 3, 4, -1/2, -3, -4, 1/2^8, 1/4, 1/8, 1/2^27, -1/2^8, -1/16, -1/2^27]
// (zkf-metal/src/poseidon2/babybear.rs:14-58) applied with additions and shifts:
// x * 2^-k = (x >> k) - (x mod 2^k) * 15 * 2^(27-k)  (mod p), because 2^-27 = -15 (mod p).
// This moves work from the integer multiplier (the binding pipe) to the ALU.
namespace bb16 {
using B = BabyBear;

__host__ __device__ __forceinline__ uint32_t sbox(uint32_t x) {
  uint32_t x2 = B::mont_lazy(x, x);             // < 2p
  uint32_t x3 = B::red(B::mont_lazy(x2, x));    // < p
  uint32_t x4 = B::mont_lazy(x2, B::red(x2));   // < 2p
  return B::red(B::mont_lazy(x4, x3));
}

template <int K>
__host__ __device__ __forceinline__ uint32_t div2k(uint32_t x) {
  return B::sub(x >> K, (x & ((1u << K) - 1u)) * (15u << (27 - K)));
}

__host__ __device__ __forceinline__ uint32_t dbl(uint32_t x) { return B::add(x, x); }

__host__ __device__ __forceinline__ void internal_round(uint32_t (&s)[16], uint32_t rc) {
  s[0] = sbox(B::add(s[0], rc));
  uint32_t sum = s[0];
#pragma unroll
  for (int i = 1; i < 16; i++) sum = B::add(sum, s[i]);
  s[0] = B::sub(sum, dbl(s[0]));
  s[1] = B::add(sum, s[1]);
  s[2] = B::add(sum, dbl(s[2]));
  s[3] = B::add(sum, div2k<1>(s[3]));
  s[4] = B::add(sum, B::add(dbl(s[4]), s[4]));
  s[5] = B::add(sum, dbl(dbl(s[5])));
  s[6] = B::sub(sum, div2k<1>(s[6]));
  s[7] = B::sub(sum, B::add(dbl(s[7]), s[7]));
  s[8] = B::sub(sum, dbl(dbl(s[8])));
  s[9] = B::add(sum, div2k<8>(s[9]));
  s[10] = B::add(sum, div2k<2>(s[10]));
  s[11] = B::add(sum, div2k<3>(s[11]));
  s[12] = B::add(sum, div2k<27>(s[12]));
  s[13] = B::sub(sum, div2k<8>(s[13]));
  s[14] = B::sub(sum, div2k<4>(s[14]));
  s[15] = B::sub(sum, div2k<27>(s[15]));
}

__host__ __device__ __forceinline__ void full_round(uint32_t (&s)[16], const uint32_t *rc) {
#pragma unroll
  for (int i = 0; i < 16; i++) s[i] = sbox(B::add(s[i], rc[i]));
  p2_ext_mds<BabyBear, 16>(s);
}

__host__ __device__ __forceinline__ void permute(uint32_t (&s)[16], const P2Params<BabyBear, 16> &p) {
  const int half = p.rounds_f / 2, rp = p.rounds_p;
  p2_ext_mds<BabyBear, 16>(s);
#pragma unroll 1
  for (int r = 0; r < half; r++) full_round(s, p.rc + r * 16);
#pragma unroll 1
  for (int r = 0; r < rp; r++) internal_round(s, p.rc[half * 16 + r]);
#pragma unroll 1
  for (int r = 0; r < half; r++) full_round(s, p.rc + half * 16 + rp + r * 16);
}
}  // namespace bb16

// The round loops are deliberately not unrolled: one full-round body (16 S-boxes + MDS,
// ~9 KB of SASS for BabyBear) and one partial-round body keep the permutation inside
// the instruction cache while many warps run it at different offsets.  Constants are
// read from the parameter bank with a per-round index (LDC, uniform across the warp).
template <class F, int W>
__host__ __device__ __forceinline__ void p2_permute(typename F::T (&s)[W], const P2Params<F, W> &p) {
  if constexpr (std::is_same<F, BabyBear>::value && W == 16) {
    if (p.diag_kind == 1) {
      bb16::permute(s, p);
      return;
    }
  }
  const int half = p.rounds_f / 2, rp = p.rounds_p;
  p2_ext_mds<F, W>(s);
#pragma unroll 1
  for (int r = 0; r < half; r++) p2_full_round<F, W>(s, p.rc + r * W);
#pragma unroll 1
  for (int r = 0; r < rp; r++) p2_partial_round<F, W>(s, p.rc[half * W + r], p.diag);
#pragma unroll 1
  for (int r = 0; r < half; r++) p2_full_round<F, W>(s, p.rc + half * W + rp + r * W);
}

}  // namespace zkb
