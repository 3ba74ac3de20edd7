// ntt_tile.cuh — the CTA-tiles of the NTT passes and of the fused LDE middle, as device
// functions: the standalone kernels of ntt.cu run one tile per block, the persistent
// batch kernel (persist.cu) runs them as work items.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <type_traits>
#include <utility>
#include <vector>

#include "field.cuh"

namespace zkb {

// -------------------------------------------------------------- pass kernel
// One pass handles index bits [lo, lo+K) of every transform: for each fixed value of
// the other bits (a "group") and each chunk of C columns, one CTA computes the
// 2^K-point sub-DFT as a four-step inside the CTA:
//   phase A: thread (i, c) loads the R1 = 2^LR1 elements x[j*R2 + i] of column c and
//            runs an R1-point DIF in registers, multiplies by w_{2^K}^{i*f1} and
//            writes them to shared memory, f1-major;
//   phase B: thread (f1, c) reads its R2 = 2^LR2 values, runs an R2-point DIF in
//            registers, applies the pass twist w_{2^hi}^{(row mod 2^lo)*f} (or the
//            final 1/n scale) and stores at the bit-reversed tile position
//            rev(f1)*R2 + t.
// Register DIFs use compile-time indices and a 32-entry table of w_64 powers passed
// as a kernel parameter, so a butterfly is one Montgomery multiply plus two adds.
struct PassGeom {
  int L;                     // log2 of each transform
  int lo;                    // lowest index bit of this pass
  uint32_t width;            // matrix columns
  uint32_t chunks_per_row;   // width / C
  uint32_t groups;           // 2^(L-K) groups per transform
  uint64_t block_stride;     // elements between transforms
  int twist;
};

// w_64^e, e < 32, for the register DIFs: BabyBear holds the canonical powers and their
// Shoup quotients (products by these constants are Shoup products), Goldilocks the
// canonical powers (q unused).
template <class F>
struct SmallTw {
  typename F::T w[32];
  typename F::T q[32];
};

// A twiddle staged in shared memory, in the form the kernels multiply by.  The cached
// tables keep the field's encoded form (Montgomery for BabyBear); staging turns a BabyBear
// entry into its canonical value and Shoup quotient, so every product by it is a Shoup
// product (about 1.5x the throughput of a Montgomery product on the integer pipes).
template <class F>
struct TwS;
template <>
struct TwS<BabyBear> {
  uint32_t w, q;
};
template <>
struct TwS<Goldilocks> {
  uint64_t w;
};

// floor(2^64 / p) for BabyBear is 2 * 2^32 + BB_RECIP_LO.
constexpr uint32_t BB_RECIP_LO = 0x2222221du;

template <class F>
__device__ __forceinline__ TwS<F> tw_stage(typename F::T enc);
template <>
__device__ __forceinline__ TwS<BabyBear> tw_stage<BabyBear>(uint32_t enc) {
  const uint32_t w = BabyBear::from_mont(enc);
  // 2w + hi(w * BB_RECIP_LO) = floor(w * floor(2^64/p) / 2^32) is floor(w 2^32 / p) or one
  // less; the remainder w 2^32 - q p is below 2p < 2^32, so its value mod 2^32 decides.
  uint32_t q = 2 * w + __umulhi(w, BB_RECIP_LO);
  if (0u - q * BabyBear::P >= BabyBear::P) q++;
  return {w, q};
}
template <>
__device__ __forceinline__ TwS<Goldilocks> tw_stage<Goldilocks>(uint64_t enc) {
  return {enc};
}

template <class F>
__device__ __forceinline__ typename F::T tw_mul(typename F::T x, const TwS<F> &t);
template <>
__device__ __forceinline__ uint32_t tw_mul<BabyBear>(uint32_t x, const TwS<BabyBear> &t) {
  return BabyBear::mul_shoup(x, t.w, t.q);
}
template <>
__device__ __forceinline__ uint64_t tw_mul<Goldilocks>(uint64_t x, const TwS<Goldilocks> &t) {
  return Goldilocks::mul(x, t.w);
}

__host__ __device__ constexpr int rev_bits(int x, int bits) {
  int r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return r;
}

// (a - b) * w for the DIF butterfly; BabyBear keeps a - b + p unreduced (< 2p), which
// the Shoup product accepts.
template <class F>
__device__ __forceinline__ typename F::T dif_mul(typename F::T a, typename F::T b, typename F::T w,
                                                 typename F::T wq);
template <>
__device__ __forceinline__ uint32_t dif_mul<BabyBear>(uint32_t a, uint32_t b, uint32_t w, uint32_t wq) {
  return BabyBear::mul_shoup(a - b + BabyBear::P, w, wq);
}
template <>
__device__ __forceinline__ uint64_t dif_mul<Goldilocks>(uint64_t a, uint64_t b, uint64_t w, uint64_t) {
  return Goldilocks::mul(Goldilocks::sub(a, b), w);
}

// Compile-time loop: fn(std::integral_constant<int, I>) for I = 0..N-1, so every index
// derived from I (bit reversals, twiddle slots) is a constant expression.
template <class Fn, int... I>
__device__ __forceinline__ void sfor_impl(Fn &fn, std::integer_sequence<int, I...>) {
  (fn(std::integral_constant<int, I>{}), ...);
}
template <int N, class Fn>
__device__ __forceinline__ void sfor(Fn &&fn) {
  if constexpr (N > 0) sfor_impl(fn, std::make_integer_sequence<int, N>{});
}

// In-register radix-2 DIF of 2^LR points: natural in, x[t] = X[rev(t)] out.
template <class F, int LR>
__device__ __forceinline__ void dif_reg(typename F::T (&x)[1 << LR], const SmallTw<F> &st) {
  using T = typename F::T;
  sfor<LR>([&](auto sc) {
    constexpr int s = LR - 1 - decltype(sc)::value;
    constexpr int h = 1 << s;
    sfor<(1 << LR) / 2>([&](auto bc) {
      constexpr int b = decltype(bc)::value;
      constexpr int j = b % h, g = (b / h) * 2 * h;
      const T a = x[g + j], c = x[g + j + h];
      x[g + j] = F::add(a, c);
      if constexpr (j == 0)
        x[g + j + h] = F::sub(a, c);
      else
        x[g + j + h] = dif_mul<F>(a, c, st.w[j << (5 - s)], st.q[j << (5 - s)]);
    });
  });
}

// ---- tensor-copy (TMA) tile loads
// A pass tile can arrive in shared memory as ONE tensor copy (cp.async.bulk.tensor,
// one CTA's destination, this GPU's memory only) instead of R1 coalesced loads per thread: the
// tensor map views a column segment as 5 dimensions (column, row bits below the pass,
// the pass's bits in two parts of at most 8, the bits above it with the transform index)
// and the box is C columns x 2^K rows, so row r of the tile lands at r * C.  Completion is
// tracked by an mbarrier; every wait gives up after a bounded number of polls and raises an
// error word instead of hanging.
constexpr uint32_t TMA_WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Polls the barrier's phase `parity` at most `limit` times; false when it never completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  uint32_t done = 0;
  for (uint32_t k = 0; k < limit && !done; k++)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
  return done != 0;
}

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
      : "memory");
}

// Shared-memory geometry of a pass with C columns per CTA: f1 blocks of R2*C values,
// padded so the stride is = C (mod 32) words and phase-B warps reading several f1
// blocks hit distinct banks.
template <int LR2, int C>
struct PassSmem {
  static constexpr int BASE = C << LR2;
  static constexpr int STRIDE = BASE + ((C - (BASE % 32)) % 32 + 32) % 32;
};

// One CTA-tile of a pass (tile index `cta`, the kernel's blockIdx.x).  PERSIST: the tile
// runs inside the persistent batch kernel, whose blocks have more threads than the tile
// uses (threads from C << LR2 up only stage twiddles and meet the barriers) and whose
// inputs were written by other blocks of the same launch (read through L2, not L1).
// TMA_IN: the tile's input rows are being copied into the start of shared memory (row r
// at r * C) by a tensor copy that completes `bar`; phase A reads them there once it has
// (a wait that gives up sets *err).
template <class F, int LR1, int LR2, int C, bool PERSIST, bool TMA_IN = false>
__device__ __forceinline__ void ntt_pass_tile(const typename F::T *in, typename F::T *out, const PassGeom &g,
                                              const typename F::T *__restrict__ tw, typename F::T post_scale,
                                              const SmallTw<F> &st, uint32_t cta, unsigned char *smem_raw,
                                              uint64_t *bar = nullptr, uint32_t *err = nullptr) {
  using T = typename F::T;
  constexpr int R1 = 1 << LR1, R2 = 1 << LR2, K = LR1 + LR2;
  constexpr int S = PassSmem<LR2, C>::STRIDE;
  T *sm = reinterpret_cast<T *>(smem_raw);
  // Twiddles shared by the C columns of the CTA, staged once:
  //   tw_in[i*TP + t]  = w_{2^K}^{i * rev(t)}   (phase-A twist of output t of thread i; rows
  //                      padded to TP = R1 + 1 entries so the distinct i of a warp hit
  //                      distinct banks)
  //   tw_out[f]        = w_{2^hi}^{i_low * f}  (pass twist), or the 1/n scale on the last pass
  constexpr int TP = R1 + 1;
  TwS<F> *tw_in = reinterpret_cast<TwS<F> *>(sm + S * R1);
  TwS<F> *tw_out = tw_in + R2 * TP;

  const bool active = !PERSIST || threadIdx.x < (unsigned)(C << LR2);
  const uint32_t chunk = cta % g.chunks_per_row;
  const uint32_t rest = cta / g.chunks_per_row;
  const uint32_t grp = rest % g.groups;
  const uint32_t blk = rest / g.groups;
  const int hi = g.lo + K;
  const uint32_t i_low = grp & ((1u << g.lo) - 1u);
  const uint32_t base_row = ((grp >> g.lo) << hi) | i_low;
  const uint32_t c = threadIdx.x % C;
  const uint32_t i = threadIdx.x / C;  // < R2 for the active threads
  const bool scale_out = g.twist || post_scale != 0;

  for (uint32_t e = threadIdx.x; e < (1u << K); e += blockDim.x) {
    const uint32_t ii = e / R1, tt = e % R1;
    tw_in[ii * TP + tt] = tw_stage<F>(tw[(ii * (__brev(tt) >> (32 - LR1))) << (g.L - K)]);
    if (g.twist)
      tw_out[e] = tw_stage<F>(tw[(i_low * e) << (g.L - hi)]);  // i_low * e < 2^hi <= 2^L
    else if (post_scale)
      tw_out[e] = tw_stage<F>(post_scale);
  }

  const size_t col0 = (size_t)blk * g.block_stride + (size_t)chunk * C + c;
  const size_t rs = (size_t)g.width << g.lo;  // elements between consecutive tile rows
  T *sm_a = sm + i * C + c;                    // phase A: + f1 * S
  // ---- phase A
  {
    T x[R1];
    if (active) {
      if constexpr (TMA_IN) {
        if (!mbar_wait(bar, 0, TMA_WAIT_LIMIT)) atomicExch(err, 1u);
        const T *tp = sm + i * C + c;
#pragma unroll
        for (int j = 0; j < R1; j++) x[j] = tp[j * R2 * C];
      } else {
        const T *p = in + col0 + ((size_t)base_row * g.width) + (size_t)i * rs;
        const size_t step = rs * R2;
#pragma unroll
        for (int j = 0; j < R1; j++) {
          if constexpr (PERSIST)
            x[j] = __ldcg(p);
          else
            x[j] = *p;
          p += step;
        }
      }
      dif_reg<F, LR1>(x, st);
    }
    __syncthreads();  // tw_in staged
    if (active) {
      const TwS<F> *twi = tw_in + i * TP;
      sfor<R1>([&](auto tc) {
        constexpr int t = decltype(tc)::value;
        T v = x[t];
        if constexpr (LR2 > 0 && t != 0) v = tw_mul<F>(v, twi[t]);
        sm_a[rev_bits(t, LR1) * S] = v;
      });
    }
  }
  __syncthreads();
  if (!active) return;
  // ---- phase B
#pragma unroll 1
  for (int q = 0; q < R1 / R2; q++) {
    const uint32_t f1 = i + q * R2;
    const T *sm_b = sm + f1 * S + c;
    T y[R2];
#pragma unroll
    for (int ii = 0; ii < R2; ii++) y[ii] = sm_b[ii * C];
    dif_reg<F, LR2>(y, st);
    T *p = out + col0 + ((size_t)base_row * g.width) + (size_t)((__brev(f1) >> (32 - LR1)) * R2) * rs;
    const TwS<F> *two = tw_out + f1;
    sfor<R2>([&](auto tc) {
      constexpr int t = decltype(tc)::value;
      T v = y[t];
      if (scale_out) v = tw_mul<F>(v, two[R1 * rev_bits(t, LR2)]);
      *p = v;
      p += rs;
    });
  }
}

// Shared-memory bytes of a pass tile.
template <class F, int LR1, int LR2, int C>
constexpr size_t pass_tile_smem() {
  return (size_t)PassSmem<LR2, C>::STRIDE * (1 << LR1) * sizeof(typename F::T) +
         (size_t)(((1u << LR2) * ((1u << LR1) + 1)) + (1u << (LR1 + LR2))) * sizeof(TwS<F>);
}

// --------------------------------------------------------- fused LDE middle
// One kernel for the last pass of the inverse transform (bits [0, K), contiguous row
// blocks B), the coset twist c_m * (s w_bn^j)^m / n of every coset j, and the first pass
// of each coset's forward transform (bits [L-K, L)).  After the inverse pass the
// coefficients of block B are c[m] with m = m_hi * 2^(L-K) + m_lo, m_lo = rev(B) fixed,
// and — as the forward pass splits m_hi = j' * R2 + i exactly like the inverse pass's
// phase B holds them — each thread already has the R1 coefficients its forward phase A
// needs, so the coefficient matrix never goes back to HBM and no expand pass runs.
struct FusedGeom {
  int L;
  uint32_t width;
  uint32_t chunks_per_row;
  uint32_t blocks;   // 2^(L-K)
  int log_b;
  uint64_t n;        // 2^L
};

// One CTA-tile of the fused LDE middle (tile index `cta`); PERSIST and TMA_IN as for
// ntt_pass_tile (the tensor copy brings the 2^K rows of block B).
template <class F, int LR1, int LR2, int C, bool PERSIST, bool TMA_IN = false>
__device__ __forceinline__ void lde_fused_tile(const typename F::T *in, typename F::T *out, const FusedGeom &g,
                                               const typename F::T *__restrict__ itw,
                                               const typename F::T *__restrict__ ftw,
                                               const typename F::T *__restrict__ ctab_t,
                                               const typename F::T *__restrict__ ftw_t, const SmallTw<F> &ist,
                                               const SmallTw<F> &fst, uint32_t cta, unsigned char *smem_raw,
                                               uint64_t *bar = nullptr, uint32_t *err = nullptr) {
  using T = typename F::T;
  constexpr int R1 = 1 << LR1, R2 = 1 << LR2, K = LR1 + LR2, Q = R1 / R2;
  constexpr int S = PassSmem<LR2, C>::STRIDE;
  T *sm = reinterpret_cast<T *>(smem_raw);
  constexpr int TP = R1 + 1;  // padded [i][t] rows: the distinct i of a warp hit distinct banks
  TwS<F> *itw_in = reinterpret_cast<TwS<F> *>(sm + S * R1);  // [i][t] inverse inner twist
  TwS<F> *ftw_in = itw_in + R2 * TP;                         // [i][t] forward inner twist
  TwS<F> *ftw_out = ftw_in + R2 * TP;                        // w_{2^L}^{m_lo * f}
  TwS<F> *cf = ftw_out + (1 << K);                           // coset factors of the current coset

  const bool active = !PERSIST || threadIdx.x < (unsigned)(C << LR2);
  const uint32_t chunk = cta % g.chunks_per_row;
  const uint32_t B = cta / g.chunks_per_row;
  const int lm = g.L - K;  // bits of m_lo
  const uint32_t m_lo = lm ? (__brev(B) >> (32 - lm)) : 0u;
  const uint32_t c = threadIdx.x % C;
  const uint32_t i = threadIdx.x / C;

  for (uint32_t e = threadIdx.x; e < (1u << K); e += blockDim.x) {
    const uint32_t ii = e / R1, tt = e % R1;
    const uint32_t ex = (ii * (__brev(tt) >> (32 - LR1))) << lm;
    itw_in[ii * TP + tt] = tw_stage<F>(itw[ex]);
    ftw_in[ii * TP + tt] = tw_stage<F>(ftw[ex]);
    ftw_out[e] = tw_stage<F>(ftw_t[((size_t)m_lo << K) + e]);  // w^(m_lo * e), contiguous per m_lo
  }

  const size_t colc = (size_t)chunk * C + c;
  T *sm_a = sm + i * C + c;
  // ---- inverse pass over the contiguous block B (no twist: lowest bits)
  T coef[R1];
  {
    T x[R1];
    if (active) {
      if constexpr (TMA_IN) {
        if (!mbar_wait(bar, 0, TMA_WAIT_LIMIT)) atomicExch(err, 1u);
        const T *tp = sm + i * C + c;
#pragma unroll
        for (int j = 0; j < R1; j++) x[j] = tp[j * R2 * C];
      } else {
        const T *p = in + colc + ((size_t)B * (1u << K) + i) * g.width;
        const size_t step = (size_t)R2 * g.width;
#pragma unroll
        for (int j = 0; j < R1; j++) {
          if constexpr (PERSIST)
            x[j] = __ldcg(p);
          else
            x[j] = *p;
          p += step;
        }
      }
      dif_reg<F, LR1>(x, ist);
    }
    __syncthreads();
    if (active) {
      const TwS<F> *twi = itw_in + i * TP;
      sfor<R1>([&](auto tc) {
        constexpr int t = decltype(tc)::value;
        T v = x[t];
        if constexpr (LR2 > 0 && t != 0) v = tw_mul<F>(v, twi[t]);
        sm_a[rev_bits(t, LR1) * S] = v;
      });
    }
  }
  __syncthreads();
  if (active) {
    sfor<Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const T *sm_b = sm + (i + q * R2) * S + c;
      T y[R2];
#pragma unroll
      for (int ii = 0; ii < R2; ii++) y[ii] = sm_b[ii * C];
      dif_reg<F, LR2>(y, ist);
      sfor<R2>([&](auto tc) {
        constexpr int t = decltype(tc)::value;
        coef[rev_bits(t, LR2) * Q + q] = y[t];
      });
    });
  }
  // ---- per coset: twist, forward pass over bits [L-K, L)
  const size_t rs = (size_t)g.width << lm;
  for (int jc = 0; jc < (1 << g.log_b); jc++) {
    __syncthreads();  // previous users of the tile and of cf are done
    // factors of m = m_lo + e * 2^lm, stored contiguously per (coset, m_lo)
    const T *ct = ctab_t + (uint64_t)jc * g.n + ((size_t)m_lo << K);
    for (uint32_t e = threadIdx.x; e < (1u << K); e += blockDim.x) cf[e] = tw_stage<F>(ct[e]);
    __syncthreads();
    if (active) {
      T x[R1];
#pragma unroll
      for (int j = 0; j < R1; j++) x[j] = tw_mul<F>(coef[j], cf[j * R2 + i]);
      dif_reg<F, LR1>(x, fst);
      const TwS<F> *twi = ftw_in + i * TP;
      sfor<R1>([&](auto tc) {
        constexpr int t = decltype(tc)::value;
        T v = x[t];
        if constexpr (LR2 > 0 && t != 0) v = tw_mul<F>(v, twi[t]);
        sm_a[rev_bits(t, LR1) * S] = v;
      });
    }
    __syncthreads();
    if (active) {
      const uint32_t r = g.log_b ? (__brev((uint32_t)jc) >> (32 - g.log_b)) : 0u;
      T *blk = out + (uint64_t)r * g.n * g.width + colc + (size_t)m_lo * g.width;
#pragma unroll 1
      for (int q = 0; q < Q; q++) {
        const uint32_t f1 = i + q * R2;
        const T *sm_b = sm + f1 * S + c;
        T y[R2];
#pragma unroll
        for (int ii = 0; ii < R2; ii++) y[ii] = sm_b[ii * C];
        dif_reg<F, LR2>(y, fst);
        T *p = blk + (size_t)((__brev(f1) >> (32 - LR1)) * R2) * rs;
        const TwS<F> *two = ftw_out + f1;
        sfor<R2>([&](auto tc) {
          constexpr int t = decltype(tc)::value;
          T v = y[t];
          if (lm > 0) v = tw_mul<F>(v, two[R1 * rev_bits(t, LR2)]);
          *p = v;
          p += rs;
        });
      }
    }
  }
}

// Shared-memory bytes of a fused tile.
template <class F, int LR1, int LR2, int C>
constexpr size_t fused_tile_smem() {
  return (size_t)PassSmem<LR2, C>::STRIDE * (1 << LR1) * sizeof(typename F::T) +
         (size_t)(2u * ((1u << LR2) * ((1u << LR1) + 1)) + (2u << (LR1 + LR2))) * sizeof(TwS<F>);
}

// ---- host side, for the persistent batch kernel (defined in ntt.cu)
// The register-DIF constants (w_64 powers and Shoup quotients) of either direction.
void small_twiddles_bb(bool inverse, SmallTw<BabyBear> *out);
// The pass split and the device tables of one BabyBear coset LDE (shift = the field
// generator, rows bit-reversed), as ntt_lde_dev runs it with passes of at most kmax bits:
// ks = pass bits top first (the last is the fused kernel's); the tables are built on s
// when missing (not inside a graph capture).
struct LdePlanBB {
  std::vector<int> ks;
  const uint32_t *itw = nullptr, *ftw = nullptr, *ctab_t = nullptr, *ftw_t = nullptr;
};
int lde_plan_babybear(int log_h, int log_b, int kmax, LdePlanBB *out, cudaStream_t s);

}  // namespace zkb
