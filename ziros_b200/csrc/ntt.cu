// ntt.cu — column-batched NTT and coset low-degree extension on row-major matrices.
//
// Reference path: MetalDft::dft_batch / idft_batch (zkf-metal/src/ntt/p3_adapter.rs:69-459)
// and p3's default coset_lde_batch + the PCS's bit_reverse_rows
// (zkf-backends/src/plonky3.rs:250-262, stark_to_groth16.rs:2324-2346).  The
// reference runs one HBM pass per radix-2 stage after a host bit-reversal; here a
// transform of size 2^L is cut into a few passes of 2^k-point sub-DFTs staged in
// shared memory (four-step decomposition, applied recursively):
//
//   pass over index bits [lo, hi):  for every fixed value of the other bits, the
//   2^k elements x[t] at rows base + t*2^lo get Y[f] = sum_t x[t] w_{2^k}^{tf}
//   (radix-2 decimation in frequency, natural in / bit-reversed out), then the
//   twist Y[f] *= w_{2^hi}^{(row mod 2^lo) * f}, stored back at rows
//   base + rev_k(f)*2^lo.
//
// Passes run from the top bits down, so the final layout is the bit-reversed
// (natural-in, reversed-out) DFT.  That is exactly the row order the PCS commits,
// so the LDE needs no separate bit-reversal:
//
//   LDE_bitrev[r*n + q] = DFT_n( c_m * (s * w_{bn}^{j})^m )[rev(q)],  j = rev_b(r),
//
// i.e. b independent size-n NR transforms of the coefficients twisted per coset.
#include <algorithm>

#include "common.cuh"
#include "engine.cuh"
#include "field.cuh"

namespace zkb {

// ------------------------------------------------------------------ tables
template <class F>
struct PowParams {
  typename F::T b2[40];  // encoded base^(2^j)
  typename F::T scale;   // encoded
};

// out[t] = scale * base^t (encoded domain), product of the base^(2^j) for the set bits of t.
template <class F>
__global__ void powers_kernel(typename F::T *out, uint64_t n, const __grid_constant__ PowParams<F> pp) {
  using D = Dom<F>;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (uint64_t)gridDim.x * blockDim.x) {
    typename F::T acc = pp.scale;
    uint64_t e = t;
    int j = 0;
    while (e) {
      if (e & 1) acc = D::mul(acc, pp.b2[j]);
      e >>= 1;
      j++;
    }
    out[t] = acc;
  }
}

template <class F>
static int launch_powers(typename F::T *out, uint64_t n, typename F::T base, typename F::T scale,
                         cudaStream_t s) {
  PowParams<F> pp;
  typename F::T b = base;
  for (int j = 0; j < 40; j++) {
    pp.b2[j] = Dom<F>::encode(b);
    b = F::mul_host(b, b);
  }
  pp.scale = Dom<F>::encode(scale);
  ZKB_LAUNCH("table_powers", s, powers_kernel<F><<<grid_for(n, 256), 256, 0, s>>>(out, n, pp));
  ZKB_CHECK_LAUNCH();
  return ZKB_OK;
}

template <class F>
static constexpr int field_id() {
  return sizeof(typename F::T) == 4 ? ZKB_FIELD_BABYBEAR : ZKB_FIELD_GOLDILOCKS;
}

template <class F>
int get_twiddles(int log_n, bool inverse, const typename F::T **out, cudaStream_t s) {
  using T = typename F::T;
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));
  if (log_n > F::TWO_ADICITY) {
    set_error("NTT size 2^%d exceeds the two-adicity of the field", log_n);
    return ZKB_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto key = std::make_tuple(field_id<F>(), log_n, (int)inverse);
  auto it = ctx->twiddles.find(key);
  if (it != ctx->twiddles.end()) {
    *out = (const T *)it->second.ptr;
    return ZKB_OK;
  }
  uint64_t n = 1ull << log_n;
  void *p = nullptr;
  ZKB_CHECK_CUDA(cudaMalloc(&p, n * sizeof(T)));
  T w = two_adic_generator<F>(log_n);
  if (inverse) w = inv_host<F>(w);
  int rc = launch_powers<F>((T *)p, n, w, 1, s);
  if (rc == ZKB_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = ZKB_ERR_CUDA;
  if (rc != ZKB_OK) {
    cudaFree(p);
    return rc;
  }
  ctx->twiddles[key] = DeviceTable{p, n * sizeof(T)};
  *out = (const T *)p;
  return ZKB_OK;
}

// Coset factors: tab[j*n + m] = (shift * w_{bn}^j)^m / n, encoded.
template <class F>
static int get_coset_table(int log_n, int log_b, typename F::T shift, const typename F::T **out,
                           cudaStream_t s) {
  using T = typename F::T;
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto key = std::make_tuple(field_id<F>(), log_n, log_b, (uint64_t)shift);
  auto it = ctx->cosets.find(key);
  if (it != ctx->cosets.end()) {
    *out = (const T *)it->second.ptr;
    return ZKB_OK;
  }
  uint64_t n = 1ull << log_n, b = 1ull << log_b;
  void *p = nullptr;
  ZKB_CHECK_CUDA(cudaMalloc(&p, n * b * sizeof(T)));
  T w_bn = two_adic_generator<F>(log_n + log_b);
  T n_inv = inv_host<F>((T)(n % (uint64_t)F::P));
  T wj = 1;
  int rc = ZKB_OK;
  for (uint64_t j = 0; j < b && rc == ZKB_OK; j++) {
    rc = launch_powers<F>((T *)p + j * n, n, F::mul_host(shift, wj), n_inv, s);
    wj = F::mul_host(wj, w_bn);
  }
  if (rc == ZKB_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = ZKB_ERR_CUDA;
  if (rc != ZKB_OK) {
    cudaFree(p);
    return rc;
  }
  ctx->cosets[key] = DeviceTable{p, n * b * sizeof(T)};
  *out = (const T *)p;
  return ZKB_OK;
}

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
  uint32_t cols;             // columns per CTA (power of two dividing width)
  int log_cols;
  uint32_t chunks_per_row;   // width / cols
  uint32_t groups;           // 2^(L-K) groups per transform
  uint32_t sm_stride;        // shared-memory stride between f1 blocks (elements)
  uint64_t block_stride;     // elements between transforms
  int twist;
};

template <class F>
struct SmallTw {
  typename F::T w[32];  // w_64^e, e < 32, encoded for F::mul_tw
};

__host__ __device__ constexpr uint32_t rev_bits(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

// (a - b) * w for the DIF butterfly; BabyBear keeps a - b + p unreduced (< 2p), which
// the lazy Montgomery product accepts.
template <class F>
__device__ __forceinline__ typename F::T dif_mul(typename F::T a, typename F::T b, typename F::T w);
template <>
__device__ __forceinline__ uint32_t dif_mul<BabyBear>(uint32_t a, uint32_t b, uint32_t w) {
  return BabyBear::red(BabyBear::mont_lazy(a - b + BabyBear::P, w));
}
template <>
__device__ __forceinline__ uint64_t dif_mul<Goldilocks>(uint64_t a, uint64_t b, uint64_t w) {
  return Goldilocks::mul(Goldilocks::sub(a, b), w);
}

// In-register radix-2 DIF of 2^LR points: natural in, x[t] = X[rev(t)] out.
template <class F, int LR>
__device__ __forceinline__ void dif_reg(typename F::T (&x)[1 << LR], const typename F::T *w64) {
  using T = typename F::T;
  constexpr int R = 1 << LR;
#pragma unroll
  for (int s = LR - 1; s >= 0; s--) {
    const int h = 1 << s;
#pragma unroll
    for (int g = 0; g < R; g += 2 * h) {
#pragma unroll
      for (int j = 0; j < h; j++) {
        T a = x[g + j], b = x[g + j + h];
        x[g + j] = F::add(a, b);
        x[g + j + h] = j == 0 ? F::sub(a, b) : dif_mul<F>(a, b, w64[j << (5 - s)]);
      }
    }
  }
}

template <class F, int LR1, int LR2>
__global__ void __launch_bounds__(512)
    ntt_pass_kernel(const typename F::T *in, typename F::T *out, const PassGeom g,
                    const typename F::T *__restrict__ tw, typename F::T post_scale,
                    const __grid_constant__ SmallTw<F> st) {
  using T = typename F::T;
  constexpr int R1 = 1 << LR1, R2 = 1 << LR2, K = LR1 + LR2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  // Twiddles shared by the C columns of the CTA, staged once:
  //   tw_in[e]  = w_{2^K}^e            (phase-A twist, e = i * f1 < 2^K)
  //   tw_out[f] = w_{2^hi}^{i_low * f} (pass twist), or the 1/n scale on the last pass
  T *tw_in = sm + (size_t)g.sm_stride * R1;
  T *tw_out = tw_in + (1 << K);

  const uint32_t cta = blockIdx.x;
  const uint32_t chunk = cta % g.chunks_per_row;
  const uint32_t rest = cta / g.chunks_per_row;
  const uint32_t grp = rest % g.groups;
  const uint32_t blk = rest / g.groups;
  const int hi = g.lo + K;
  const uint32_t i_low = grp & ((1u << g.lo) - 1u);
  const uint32_t base_row = ((grp >> g.lo) << hi) | i_low;
  const uint32_t lc = g.log_cols;
  const uint32_t c = threadIdx.x & (g.cols - 1);
  const uint32_t i = threadIdx.x >> lc;  // < R2
  const bool scale_out = g.twist || post_scale != 0;

  for (uint32_t e = threadIdx.x; e < (1u << K); e += blockDim.x) {
    tw_in[e] = tw[e << (g.L - K)];
    if (g.twist)
      tw_out[e] = tw[(i_low * e) << (g.L - hi)];  // i_low * e < 2^hi <= 2^L
    else if (post_scale)
      tw_out[e] = post_scale;
  }

  const size_t col0 = (size_t)blk * g.block_stride + (size_t)chunk * g.cols + c;
  const size_t rs = (size_t)g.width << g.lo;  // elements between consecutive tile rows
  // ---- phase A
  {
    T x[R1];
    const T *p = in + col0 + ((size_t)base_row * g.width) + (size_t)i * rs;
    const size_t step = rs * R2;
#pragma unroll
    for (int j = 0; j < R1; j++) {
      x[j] = *p;
      p += step;
    }
    dif_reg<F, LR1>(x, st.w);
    __syncthreads();  // tw_in staged
#pragma unroll
    for (int t = 0; t < R1; t++) {
      const uint32_t f1 = rev_bits((uint32_t)t, LR1);
      T v = x[t];
      if (LR2 > 0 && f1 != 0) v = F::mul_tw(v, tw_in[i * f1]);
      sm[f1 * g.sm_stride + (i << lc) + c] = v;
    }
  }
  __syncthreads();
  // ---- phase B
#pragma unroll 1
  for (int q = 0; q < R1 / R2; q++) {
    const uint32_t f1 = i + q * R2;
    T y[R2];
#pragma unroll
    for (int ii = 0; ii < R2; ii++) y[ii] = sm[f1 * g.sm_stride + (ii << lc) + c];
    dif_reg<F, LR2>(y, st.w);
    T *p = out + col0 + ((size_t)base_row * g.width) + (size_t)(rev_bits(f1, LR1) * R2) * rs;
#pragma unroll
    for (int t = 0; t < R2; t++) {
      T v = y[t];
      if (scale_out) v = F::mul_tw(v, tw_out[f1 + R1 * rev_bits((uint32_t)t, LR2)]);
      *p = v;
      p += rs;
    }
  }
}

template <class F>
static uint32_t pick_cols(uint32_t width) {
  uint32_t cmax = sizeof(typename F::T) == 4 ? 16 : 8;
  uint32_t c = 1;
  while (c * 2 <= cmax && width % (c * 2) == 0) c *= 2;
  return c;
}

// Split L bits into passes of at most kmax bits, as even as possible, top first.
static std::vector<int> plan_passes(int L, int kmax) {
  std::vector<int> ks;
  if (L <= 0) return ks;
  int np = (L + kmax - 1) / kmax;
  for (int i = 0; i < np; i++) ks.push_back(L / np + (i < L % np ? 1 : 0));
  return ks;
}

template <class F>
static SmallTw<F> small_twiddles(bool inverse) {
  SmallTw<F> st;
  typename F::T w = two_adic_generator<F>(6), acc = 1;
  if (inverse) w = inv_host<F>(w);
  for (int e = 0; e < 32; e++) {
    st.w[e] = Dom<F>::encode(acc);
    acc = F::mul_host(acc, w);
  }
  return st;
}

template <class F, int LR1, int LR2>
static int launch_pass(const typename F::T *src, typename F::T *out, const PassGeom &g, uint64_t ctas,
                       const typename F::T *tw, typename F::T scale, const SmallTw<F> &st,
                       cudaStream_t s) {
  using T = typename F::T;
  const unsigned threads = g.cols << LR2;
  const size_t smem = (((size_t)g.sm_stride << LR1) + (2u << (LR1 + LR2))) * sizeof(T);
  ZKB_CHECK_CUDA(cudaFuncSetAttribute(ntt_pass_kernel<F, LR1, LR2>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  ZKB_LAUNCH("ntt_pass", s, ntt_pass_kernel<F, LR1, LR2><<<(unsigned)ctas, threads, smem, s>>>(src, out, g, tw, scale, st));
  return ZKB_OK;
}

template <class F>
static int run_passes(const typename F::T *in, typename F::T *out, int L, uint32_t width,
                      uint64_t n_blocks, const typename F::T *tw, bool inverse,
                      typename F::T last_scale, cudaStream_t s) {
  using T = typename F::T;
  const uint32_t C = pick_cols<F>(width);
  int lc = 0;
  while ((1u << lc) < C) lc++;
  // BabyBear: up to 64 + 32 registers of data per thread phase; Goldilocks: 32 + 32.
  const int kmax = sizeof(T) == 4 ? 11 : 10;
  std::vector<int> ks = plan_passes(L, kmax);
  // the register DIFs use w_64 of the same direction as the table `tw`
  const SmallTw<F> st = small_twiddles<F>(inverse);
  int hi = L;
  const T *src = in;
  for (size_t pi = 0; pi < ks.size(); pi++) {
    const int K = ks[pi];
    PassGeom g;
    g.L = L;
    g.lo = hi - K;
    g.width = width;
    g.cols = C;
    g.log_cols = lc;
    g.chunks_per_row = width / C;
    g.groups = 1u << (L - K);
    // stride between f1 blocks = R2*C padded to = C (mod 32) elements: the warps of
    // phase B read two or more f1 blocks at once without bank conflicts
    uint32_t base = C << (K / 2);
    g.sm_stride = base + ((C - (base % 32u)) % 32u);
    g.block_stride = ((uint64_t)width) << L;
    g.twist = g.lo > 0;
    const uint64_t ctas = (uint64_t)g.chunks_per_row * g.groups * n_blocks;
    if (ctas >= (1ull << 31) || ((uint64_t)width << L) * n_blocks >= (1ull << 40)) {
      set_error("NTT launch too large");
      return ZKB_ERR_UNSUPPORTED;
    }
    const T scale = (pi + 1 == ks.size()) ? last_scale : (T)0;
    int rc;
    switch (K) {
      case 1: rc = launch_pass<F, 1, 0>(src, out, g, ctas, tw, scale, st, s); break;
      case 2: rc = launch_pass<F, 1, 1>(src, out, g, ctas, tw, scale, st, s); break;
      case 3: rc = launch_pass<F, 2, 1>(src, out, g, ctas, tw, scale, st, s); break;
      case 4: rc = launch_pass<F, 2, 2>(src, out, g, ctas, tw, scale, st, s); break;
      case 5: rc = launch_pass<F, 3, 2>(src, out, g, ctas, tw, scale, st, s); break;
      case 6: rc = launch_pass<F, 3, 3>(src, out, g, ctas, tw, scale, st, s); break;
      case 7: rc = launch_pass<F, 4, 3>(src, out, g, ctas, tw, scale, st, s); break;
      case 8: rc = launch_pass<F, 4, 4>(src, out, g, ctas, tw, scale, st, s); break;
      case 9: rc = launch_pass<F, 5, 4>(src, out, g, ctas, tw, scale, st, s); break;
      case 10: rc = launch_pass<F, 5, 5>(src, out, g, ctas, tw, scale, st, s); break;
      case 11:
        if constexpr (sizeof(T) == 4) {
          rc = launch_pass<F, 6, 5>(src, out, g, ctas, tw, scale, st, s);
          break;
        }
        [[fallthrough]];
      default:
        set_error("internal: NTT pass of %d bits", K);
        return ZKB_ERR_INTERNAL;
    }
    ZKB_TRY(rc);
    src = out;
    hi = g.lo;
  }
  return ZKB_OK;
}

// ------------------------------------------------------- auxiliary kernels
template <class F>
__global__ void bitrev_rows_kernel(const typename F::T *__restrict__ in, typename F::T *__restrict__ out,
                                   int L, uint32_t width, uint64_t total) {
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t row = idx / width, c = idx - row * width;
    uint64_t r = L ? (__brevll(row) >> (64 - L)) : 0;
    out[r * width + c] = in[idx];
  }
}

// Coefficients in bit-reversed row order -> b twisted copies in natural order.
template <class F>
__global__ void lde_expand_kernel(const typename F::T *__restrict__ coef, typename F::T *__restrict__ out,
                                  int L, int log_b, uint32_t width,
                                  const typename F::T *__restrict__ ctab) {
  const uint64_t n = 1ull << L, total = n * width;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t m = idx / width, c = idx - m * width;
    uint64_t src = L ? (__brevll(m) >> (64 - L)) : 0;
    typename F::T v = coef[src * width + c];
    for (uint32_t r = 0; r < (1u << log_b); r++) {
      uint32_t j = log_b ? (__brev(r) >> (32 - log_b)) : 0;
      out[(((uint64_t)r << L) + m) * width + c] = F::mul_tw(v, ctab[((uint64_t)j << L) + m]);
    }
  }
}

// ----------------------------------------------------------------- drivers
template <class F>
int ntt_dft_dev(typename F::T *d, int log_h, uint32_t width, bool inverse, cudaStream_t s) {
  using T = typename F::T;
  if (width == 0 || log_h == 0) return ZKB_OK;
  const T *tw;
  ZKB_TRY(get_twiddles<F>(log_h, inverse, &tw, s));
  uint64_t n = 1ull << log_h;
  ScratchBuf tmp;
  ZKB_TRY(tmp.alloc(n * width * sizeof(T), s));
  T scale = 0;
  if (inverse) scale = Dom<F>::encode(inv_host<F>((T)(n % (uint64_t)F::P)));
  ZKB_TRY(run_passes<F>(d, tmp.as<T>(), log_h, width, 1, tw, inverse, scale, s));
  ZKB_LAUNCH("bitrev_rows", s, bitrev_rows_kernel<F><<<grid_for(n * width, 256), 256, 0, s>>>(tmp.as<T>(), d, log_h, width,
                                                                   n * width));
  ZKB_CHECK_LAUNCH();
  return ZKB_OK;
}

template <class F>
int ntt_lde_dev(const typename F::T *d_trace, int log_h, uint32_t width, int log_b,
                typename F::T shift, bool bitrev, typename F::T *d_out, cudaStream_t s) {
  using T = typename F::T;
  if (width == 0) return ZKB_OK;
  if (log_h + log_b > F::TWO_ADICITY) {
    set_error("LDE size 2^%d exceeds the two-adicity of the field", log_h + log_b);
    return ZKB_ERR_INVALID;
  }
  const uint64_t n = 1ull << log_h;
  ScratchBuf coef;
  ZKB_TRY(coef.alloc(n * width * sizeof(T), s));
  if (log_h > 0) {
    const T *itw;
    ZKB_TRY(get_twiddles<F>(log_h, true, &itw, s));
    ZKB_TRY(run_passes<F>(d_trace, coef.as<T>(), log_h, width, 1, itw, true, (T)0, s));
  } else {
    ZKB_CHECK_CUDA(cudaMemcpyAsync(coef.p, d_trace, width * sizeof(T), cudaMemcpyDeviceToDevice, s));
  }
  const T *ctab;
  ZKB_TRY(get_coset_table<F>(log_h, log_b, shift, &ctab, s));
  ZKB_LAUNCH("lde_expand", s, lde_expand_kernel<F><<<grid_for(n * width, 256), 256, 0, s>>>(coef.as<T>(), d_out, log_h, log_b,
                                                                  width, ctab));
  ZKB_CHECK_LAUNCH();
  if (log_h > 0) {
    const T *tw;
    ZKB_TRY(get_twiddles<F>(log_h, false, &tw, s));
    ZKB_TRY(run_passes<F>(d_out, d_out, log_h, width, 1ull << log_b, tw, false, (T)0, s));
  }
  if (!bitrev) {
    const int LN = log_h + log_b;
    const uint64_t total = (n << log_b) * width;
    ScratchBuf tmp;
    ZKB_TRY(tmp.alloc(total * sizeof(T), s));
    ZKB_LAUNCH("bitrev_rows", s, bitrev_rows_kernel<F><<<grid_for(total, 256), 256, 0, s>>>(d_out, tmp.as<T>(), LN, width, total));
    ZKB_CHECK_LAUNCH();
    ZKB_CHECK_CUDA(cudaMemcpyAsync(d_out, tmp.p, total * sizeof(T), cudaMemcpyDeviceToDevice, s));
  }
  return ZKB_OK;
}

// Natural-order column DFT whose twiddle table and out-of-place temp are supplied by the
// caller (tw_buf: 2^log_h elements, tmp: 2^log_h x width elements); the table is
// regenerated into tw_buf on every call.  Used by the allocation-free entry point.
template <class F>
int ntt_dft_into(typename F::T *d, int log_h, uint32_t width, bool inverse, typename F::T *tw_buf,
                 typename F::T *tmp, cudaStream_t s) {
  using T = typename F::T;
  if (width == 0 || log_h == 0) return ZKB_OK;
  const uint64_t n = 1ull << log_h;
  T w = two_adic_generator<F>(log_h);
  if (inverse) w = inv_host<F>(w);
  ZKB_TRY(launch_powers<F>(tw_buf, n, w, 1, s));
  T scale = 0;
  if (inverse) scale = Dom<F>::encode(inv_host<F>((T)(n % (uint64_t)F::P)));
  ZKB_TRY(run_passes<F>(d, tmp, log_h, width, 1, tw_buf, inverse, scale, s));
  ZKB_LAUNCH("bitrev_rows", s, bitrev_rows_kernel<F><<<grid_for(n * width, 256), 256, 0, s>>>(tmp, d, log_h, width, n * width));
  return ZKB_OK;
}

template int ntt_dft_into<BabyBear>(uint32_t *, int, uint32_t, bool, uint32_t *, uint32_t *, cudaStream_t);
template int ntt_dft_into<Goldilocks>(uint64_t *, int, uint32_t, bool, uint64_t *, uint64_t *, cudaStream_t);

template int get_twiddles<BabyBear>(int, bool, const uint32_t **, cudaStream_t);
template int get_twiddles<Goldilocks>(int, bool, const uint64_t **, cudaStream_t);
template int ntt_dft_dev<BabyBear>(uint32_t *, int, uint32_t, bool, cudaStream_t);
template int ntt_dft_dev<Goldilocks>(uint64_t *, int, uint32_t, bool, cudaStream_t);
template int ntt_lde_dev<BabyBear>(const uint32_t *, int, uint32_t, int, uint32_t, bool, uint32_t *,
                                   cudaStream_t);
template int ntt_lde_dev<Goldilocks>(const uint64_t *, int, uint32_t, int, uint64_t, bool,
                                     uint64_t *, cudaStream_t);

}  // namespace zkb
