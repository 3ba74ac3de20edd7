// field.cuh — BabyBear and Goldilocks arithmetic for sm_100a.
//
// BabyBear (p = 2^31 - 2^27 + 1) uses 32-bit Montgomery multiplication with
// R = 2^32: four 32-bit multiplies (lo, hi, lo, hi) and a conditional add.
// Goldilocks (p = 2^64 - 2^32 + 1) uses the special-form reduction
// 2^64 = 2^32 - 1 (mod p) of the 128-bit product.
//
// Reference semantics: zkf-metal/src/shaders/field_babybear.metal:1-25 and
// field_goldilocks.metal:1-56.  Every value that leaves a kernel is canonical.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace zkb {

// ----------------------------------------------------------------- BabyBear
struct BabyBear {
  using T = uint32_t;
  static constexpr uint32_t P = 0x78000001u;
  // p^-1 mod 2^32: p = 1 + 15*2^27, so p^-1 = 1 - 15*2^27 (the square term vanishes).
  static constexpr uint32_t PINV = 0x88000001u;
  static constexpr uint32_t R2 = 0x45dddde3u;  // 2^64 mod p (to-Montgomery factor)
  static constexpr uint32_t ONE_MONT = 0x0ffffffeu;  // 2^32 mod p
  static constexpr int TWO_ADICITY = 27;
  static constexpr uint32_t GENERATOR = 31;

  static constexpr uint32_t NPINV = 0x77ffffffu;  // -p^-1 mod 2^32

  // [0, 2p) -> [0, p): the wrapped difference is larger than x exactly when x < p.
  __host__ __device__ __forceinline__ static uint32_t red(uint32_t x) {
    uint32_t y = x - P;
    return x < y ? x : y;
  }
  __host__ __device__ __forceinline__ static uint32_t add(uint32_t a, uint32_t b) { return red(a + b); }
  __host__ __device__ __forceinline__ static uint32_t sub(uint32_t a, uint32_t b) {
    uint32_t d = a - b, e = d + P;
    return d < e ? d : e;
  }
  __host__ __device__ __forceinline__ static uint32_t neg(uint32_t a) { return a ? P - a : 0; }
  // Montgomery product a*b*2^-32 in [0, 2p), for a*b < p*2^32 (one operand < 2p and the
  // other < p suffices): t = a*b, m = t*(-p^-1) mod 2^32, (t + m*p) / 2^32.  The 64-bit
  // multiply-adds map onto wide integer multiply-adds.
  __host__ __device__ __forceinline__ static uint32_t mont_lazy(uint32_t a, uint32_t b) {
    uint64_t t = (uint64_t)a * b;
    uint32_t m = (uint32_t)t * NPINV;
    uint64_t u = t + (uint64_t)m * P;
    return (uint32_t)(u >> 32);
  }
  // (a0*b0 + a1*b1) * 2^-32 in [0, 2p), for canonical operands (the sum stays below
  // 2p^2 < p*2^32): two products, one reduction.
  __host__ __device__ __forceinline__ static uint32_t mont_lazy_sum(uint32_t a0, uint32_t b0, uint32_t a1,
                                                                    uint32_t b1) {
    uint64_t t = (uint64_t)a0 * b0 + (uint64_t)a1 * b1;
    uint32_t m = (uint32_t)t * NPINV;
    uint64_t u = t + (uint64_t)m * P;
    return (uint32_t)(u >> 32);
  }
  // t * 2^-32 mod p, canonical, for any t < p*2^32 (e.g. a sum of mont_lazy results).
  __host__ __device__ __forceinline__ static uint32_t mont_reduce(uint64_t t) {
    uint32_t m = (uint32_t)t * NPINV;
    return red((uint32_t)((t + (uint64_t)m * P) >> 32));
  }
  // Fully reduced Montgomery product (both operands < p).
  __host__ __device__ __forceinline__ static uint32_t mont(uint32_t a, uint32_t b) {
    return red(mont_lazy(a, b));
  }
  __host__ __device__ __forceinline__ static uint32_t to_mont(uint32_t a) { return mont(a, R2); }
  __host__ __device__ __forceinline__ static uint32_t from_mont(uint32_t a) { return mont(a, 1); }
  // Canonical x times a twiddle stored in Montgomery form -> canonical product.
  __host__ __device__ __forceinline__ static uint32_t mul_tw(uint32_t x, uint32_t w_mont) {
    return mont(x, w_mont);
  }
  // Product by a constant w (canonical) with its Shoup quotient wq = floor(w * 2^32 / p):
  // q = floor(x * wq / 2^32) underestimates x * w / p by at most 1, so x * w - q * p,
  // computed mod 2^32, lies in [0, 2p); any x < 2^32.  Two multiplies and a multiply-add
  // against the three wide-result multiplies of a Montgomery product.
  __host__ __device__ __forceinline__ static uint32_t mul_shoup(uint32_t x, uint32_t w, uint32_t wq) {
#ifdef __CUDA_ARCH__
    const uint32_t q = __umulhi(x, wq);
#else
    const uint32_t q = (uint32_t)(((uint64_t)x * wq) >> 32);
#endif
    return red(x * w - q * P);
  }
  static inline uint32_t shoup_quotient(uint32_t w) { return (uint32_t)(((uint64_t)w << 32) / P); }
  // Host-side plain product (tables, constants).
  static inline uint32_t mul_host(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * b) % P);
  }
  // Encoding of a canonical twiddle for mul_tw.
  static inline uint32_t tw_encode(uint32_t w) { return (uint32_t)(((uint64_t)w << 32) % P); }
};

// --------------------------------------------------------------- Goldilocks
struct Goldilocks {
  using T = uint64_t;
  static constexpr uint64_t P = 0xFFFFFFFF00000001ull;
  static constexpr uint64_t EPS = 0xFFFFFFFFull;  // 2^64 - p
  static constexpr int TWO_ADICITY = 32;
  static constexpr uint64_t GENERATOR = 7;

  __host__ __device__ __forceinline__ static uint64_t canon(uint64_t x) {
    return x >= P ? x - P : x;
  }
  __host__ __device__ __forceinline__ static uint64_t add(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    // One carry chain: s = a + b (carry c), t = s + EPS (carry d).  The sum is >= p
    // exactly when c or d is set (a + b >= 2^64, or s >= 2^64 - EPS = p), and then the
    // answer is t: s - p when a + b < 2^64, and s + 2^64 - p (no second carry: s stays
    // below 2^64 - 2^33 + 1) when it overflowed.  For canonical a, b.
    uint32_t lo, hi;
    asm("{\n\t.reg .u32 s0, s1, t0, t1, c;\n\t.reg .pred q;\n\t"
        "add.cc.u32 s0, %2, %4;\n\t"
        "addc.cc.u32 s1, %3, %5;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "add.cc.u32 t0, s0, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 t1, s1, 0;\n\t"
        "addc.u32 c, c, 0;\n\t"
        "setp.ne.u32 q, c, 0;\n\t"
        "selp.u32 %0, t0, s0, q;\n\t"
        "selp.u32 %1, t1, s1, q;\n\t}"
        : "=r"(lo), "=r"(hi)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)hi << 32) | lo;
#else
    uint64_t s = a + b;
    // carry out of 2^64: 2^64 = EPS (mod p); the sum of two canonical values stays < 2^64 after it
    if (s < a) s += EPS;
    return canon(s);
#endif
  }
  __host__ __device__ __forceinline__ static uint64_t sub(uint64_t a, uint64_t b) {
    uint64_t d = a - b;
    if (a < b) d -= EPS;  // d + 2^64 - EPS = a - b + p
    return d;
  }
  __host__ __device__ __forceinline__ static uint64_t neg(uint64_t a) { return a ? P - a : 0; }
  // Reduce hi*2^64 + lo: 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
  __host__ __device__ __forceinline__ static uint64_t reduce128(uint64_t lo, uint64_t hi) {
    uint64_t hi_hi = hi >> 32, hi_lo = hi & 0xFFFFFFFFull;
    uint64_t t0 = lo - hi_hi;
    if (lo < hi_hi) t0 -= EPS;
    uint64_t t1 = hi_lo * EPS;
    uint64_t r = t0 + t1;
    if (r < t1) r += EPS;
    return canon(r);
  }
  __host__ __device__ __forceinline__ static uint64_t mul(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    // 128-bit product from four 32x32 partial products (eight 32-bit multiplies, one
    // carry chain), then the reduction with 32-bit adds/subtracts only:
    //   x = r3*2^96 + r2*2^64 + (r1:r0) = (r1:r0) - r3 + r2*(2^32 - 1)   (mod p)
    uint32_t r0, r1, r2, r3;
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    asm("mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;"
        : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
    uint32_t t0, t1, u0, u1, s0, s1;
    // t = (r1:r0) - r3, plus p on a borrow (as "- EPS": the raw difference exceeds EPS then)
    asm("{\n\t.reg .u32 m;\n\t"
        "sub.cc.u32 %0, %2, %4;\n\t"
        "subc.cc.u32 %1, %3, 0;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t}"
        : "=&r"(t0), "=&r"(t1)
        : "r"(r0), "r"(r1), "r"(r3));
    // u = r2 * 2^32 - r2 (< 2^64)
    asm("sub.cc.u32 %0, 0, %2;\n\t"
        "subc.u32 %1, %2, 0;"
        : "=&r"(u0), "=&r"(u1)
        : "r"(r2));
    // s = t + u, plus EPS on a carry out of 2^64 (2^64 = EPS mod p; no second carry)
    asm("{\n\t.reg .u32 c;\n\t"
        "add.cc.u32 %0, %2, %4;\n\t"
        "addc.cc.u32 %1, %3, %5;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"
        "add.cc.u32 %0, %0, c;\n\t"
        "addc.u32 %1, %1, 0;\n\t}"
        : "=&r"(s0), "=&r"(s1)
        : "r"(t0), "r"(t1), "r"(u0), "r"(u1));
    return canon(((uint64_t)s1 << 32) | s0);
#else
    unsigned __int128 t = (unsigned __int128)a * b;
    return reduce128((uint64_t)t, (uint64_t)(t >> 64));
#endif
  }
  __host__ __device__ __forceinline__ static uint64_t mul_tw(uint64_t x, uint64_t w) { return mul(x, w); }
  static inline uint64_t mul_host(uint64_t a, uint64_t b) { return mul(a, b); }
  static inline uint64_t tw_encode(uint64_t w) { return w; }
};

// "Encoded" domain used for twiddles, coset factors and Poseidon2 state:
// Montgomery form for BabyBear (products are single Montgomery multiplications),
// canonical for Goldilocks.
template <class F>
struct Dom;

template <>
struct Dom<BabyBear> {
  using T = uint32_t;
  __host__ __device__ __forceinline__ static T enter(T x) { return BabyBear::to_mont(x); }
  __host__ __device__ __forceinline__ static T leave(T x) { return BabyBear::from_mont(x); }
  __host__ __device__ __forceinline__ static T mul(T a, T b) { return BabyBear::mont(a, b); }
  __host__ __device__ __forceinline__ static T add(T a, T b) { return BabyBear::add(a, b); }
  __host__ __device__ __forceinline__ static T sub(T a, T b) { return BabyBear::sub(a, b); }
  static inline T encode(uint64_t canonical) { return BabyBear::tw_encode((uint32_t)canonical); }
  static constexpr T ONE = BabyBear::ONE_MONT;
};

template <>
struct Dom<Goldilocks> {
  using T = uint64_t;
  __host__ __device__ __forceinline__ static T enter(T x) { return x; }
  __host__ __device__ __forceinline__ static T leave(T x) { return x; }
  __host__ __device__ __forceinline__ static T mul(T a, T b) { return Goldilocks::mul(a, b); }
  __host__ __device__ __forceinline__ static T add(T a, T b) { return Goldilocks::add(a, b); }
  __host__ __device__ __forceinline__ static T sub(T a, T b) { return Goldilocks::sub(a, b); }
  static inline T encode(uint64_t canonical) { return canonical; }
  static constexpr T ONE = 1;
};

template <class F>
static inline typename F::T pow_host(typename F::T a, uint64_t e) {
  typename F::T r = 1, b = a;
  while (e) {
    if (e & 1) r = F::mul_host(r, b);
    b = F::mul_host(b, b);
    e >>= 1;
  }
  return r;
}
template <class F>
static inline typename F::T inv_host(typename F::T a) {
  return pow_host<F>(a, (uint64_t)F::P - 2);
}
// two_adic_generator(bits) = (g^((p-1)/2^S))^(2^(S-bits)).
template <class F>
static inline typename F::T two_adic_generator(int bits) {
  typename F::T root = pow_host<F>(F::GENERATOR, ((uint64_t)F::P - 1) >> F::TWO_ADICITY);
  for (int i = bits; i < F::TWO_ADICITY; i++) root = F::mul_host(root, root);
  return root;
}

}  // namespace zkb
