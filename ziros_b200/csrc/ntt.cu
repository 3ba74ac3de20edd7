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
#include <atomic>
#include <cstdlib>
#include <type_traits>
#include <utility>

#include "common.cuh"
#include "engine.cuh"
#include "field.cuh"
#include "ntt_tile.cuh"

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

// A cached table for use on stream s (context lock held): s waits for the table's build.
// Inside a graph capture the wait is captured as a wait on an external event, which is a
// no-op once the build has finished.
static int table_use(DeviceTable &t, cudaStream_t s) {
  if (t.complete || !t.ready) return ZKB_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ZKB_CHECK_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    ZKB_CHECK_CUDA(cudaStreamWaitEvent(s, t.ready, cudaEventWaitExternal));
    return ZKB_OK;
  }
  const cudaError_t q = cudaEventQuery(t.ready);
  if (q == cudaSuccess) {
    t.complete = true;
    return ZKB_OK;
  }
  if (q != cudaErrorNotReady) ZKB_CHECK_CUDA(q);
  ZKB_CHECK_CUDA(cudaStreamWaitEvent(s, t.ready, 0));
  return ZKB_OK;
}

// A table is built on the stream that first needs it, never inside a graph capture (the
// capture would own its memory).
static int table_build_allowed(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ZKB_CHECK_CUDA(cudaStreamIsCapturing(s, &cs));
  ZKB_REQUIRE(cs == cudaStreamCaptureStatusNone,
              "NTT tables for this shape are built on first use, which cannot happen inside a graph "
              "capture: run the shape once before capturing");
  return ZKB_OK;
}

// Table memory lives as long as the process and is allocated outside the stream-ordered
// pool, so permanent blocks do not fragment the pool that jobs allocate from and free to.
static int table_alloc(void **p, size_t bytes) {
  note_device_alloc();
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error("NTT table allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? ZKB_ERR_OOM : ZKB_ERR_CUDA;
  }
  return ZKB_OK;
}

// Publishes a table whose build was just enqueued on s.
static int table_publish(DeviceTable &t, cudaStream_t s) {
  ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&t.ready, cudaEventDisableTiming));
  ZKB_CHECK_CUDA(cudaEventRecord(t.ready, s));
  return ZKB_OK;
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
    ZKB_TRY(table_use(it->second, s));
    *out = (const T *)it->second.ptr;
    return ZKB_OK;
  }
  ZKB_TRY(table_build_allowed(s));
  uint64_t n = 1ull << log_n;
  void *p = nullptr;
  ZKB_TRY(table_alloc(&p, n * sizeof(T)));
  T w = two_adic_generator<F>(log_n);
  if (inverse) w = inv_host<F>(w);
  DeviceTable t{p, n * sizeof(T)};
  int rc = launch_powers<F>((T *)p, n, w, 1, s);
  if (rc == ZKB_OK) rc = table_publish(t, s);
  if (rc != ZKB_OK) {
    cudaFree(p);  // error path only
    return rc;
  }
  ctx->twiddles[key] = t;
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
    ZKB_TRY(table_use(it->second, s));
    *out = (const T *)it->second.ptr;
    return ZKB_OK;
  }
  ZKB_TRY(table_build_allowed(s));
  uint64_t n = 1ull << log_n, b = 1ull << log_b;
  void *p = nullptr;
  ZKB_TRY(table_alloc(&p, n * b * sizeof(T)));
  T w_bn = two_adic_generator<F>(log_n + log_b);
  T n_inv = inv_host<F>((T)(n % (uint64_t)F::P));
  T wj = 1;
  int rc = ZKB_OK;
  for (uint64_t j = 0; j < b && rc == ZKB_OK; j++) {
    rc = launch_powers<F>((T *)p + j * n, n, F::mul_host(shift, wj), n_inv, s);
    wj = F::mul_host(wj, w_bn);
  }
  DeviceTable t{p, n * b * sizeof(T)};
  if (rc == ZKB_OK) rc = table_publish(t, s);
  if (rc != ZKB_OK) {
    cudaFree(p);  // error path only
    return rc;
  }
  ctx->cosets[key] = t;
  *out = (const T *)p;
  return ZKB_OK;
}

// The fused LDE kernel's tables in the order it reads them (one contiguous run per CTA):
//   ctab_t[j*n + m_lo*2^K + e] = ctab[j*n + m_lo + e*2^(L-K)]   (coset factors)
//   ftw_t[m_lo*2^K + e]        = ftw[m_lo * e]                   (forward output twists)
template <class F>
__global__ void fused_tables_kernel(const typename F::T *__restrict__ ctab, const typename F::T *__restrict__ ftw,
                                    int L, int K, int log_b, typename F::T *__restrict__ ctab_t,
                                    typename F::T *__restrict__ ftw_t) {
  const uint64_t n = 1ull << L, nc = n << log_b, total = nc + n, mask = (1ull << K) - 1;
  for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (uint64_t)gridDim.x * blockDim.x) {
    if (idx < nc) {
      const uint64_t jc = idx >> L, r = idx & (n - 1), m_lo = r >> K, e = r & mask;
      ctab_t[idx] = ctab[(jc << L) + m_lo + (e << (L - K))];
    } else {
      const uint64_t r = idx - nc, m_lo = r >> K, e = r & mask;
      ftw_t[r] = ftw[m_lo * e];
    }
  }
}

template <class F>
static int get_fused_tables(int log_n, int log_b, typename F::T shift, int K, const typename F::T *ctab,
                            const typename F::T *ftw, const typename F::T **ctab_t, const typename F::T **ftw_t,
                            cudaStream_t s) {
  using T = typename F::T;
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto key = std::make_tuple(field_id<F>(), log_n, log_b, (uint64_t)shift, K);
  const uint64_t n = 1ull << log_n;
  auto it = ctx->fused.find(key);
  if (it == ctx->fused.end()) {
    // ctab and ftw come from get_coset_table / get_twiddles on this stream, which made s
    // wait for their builds
    ZKB_TRY(table_build_allowed(s));
    void *p = nullptr;
    ZKB_TRY(table_alloc(&p, ((n << log_b) + n) * sizeof(T)));
    T *ct = (T *)p, *ft = ct + (n << log_b);
    ZKB_LAUNCH("table_fused", s, fused_tables_kernel<F><<<grid_for((n << log_b) + n, 256), 256, 0, s>>>(ctab, ftw, log_n, K, log_b, ct, ft));
    DeviceTable t{p, ((n << log_b) + n) * sizeof(T)};
    ZKB_TRY(table_publish(t, s));
    it = ctx->fused.emplace(key, t).first;
  } else {
    ZKB_TRY(table_use(it->second, s));
  }
  *ctab_t = (const T *)it->second.ptr;
  *ftw_t = *ctab_t + (n << log_b);
  return ZKB_OK;
}

// -------------------------------------------------------------- pass kernel
// (geometry, tile code and helpers: ntt_tile.cuh)
template <class F, int LR1, int LR2, int C>
__global__ void __launch_bounds__(C << LR2)
    ntt_pass_kernel(const typename F::T *in, typename F::T *out, const PassGeom g,
                    const typename F::T *__restrict__ tw, typename F::T post_scale,
                    const __grid_constant__ SmallTw<F> st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ntt_pass_tile<F, LR1, LR2, C, false>(in, out, g, tw, post_scale, st, blockIdx.x, smem_raw);
}

// The same pass with its tile brought in by one tensor copy (see ntt_tile.cuh).  Thread 0
// sets up the barrier and issues the copy, which runs while the block stages its
// twiddles.
template <class F, int LR1, int LR2, int C>
constexpr size_t tma_bar_off() {
  return (pass_tile_smem<F, LR1, LR2, C>() + 15) & ~(size_t)15;
}

__device__ uint32_t g_tma_wait_errors;

template <class F, int LR1, int LR2, int C>
__global__ void __launch_bounds__(C << LR2)
    ntt_pass_tma_kernel(const typename F::T *in, typename F::T *out, const PassGeom g,
                        const typename F::T *__restrict__ tw, typename F::T post_scale,
                        const __grid_constant__ SmallTw<F> st, const __grid_constant__ CUtensorMap map) {
  extern __shared__ __align__(128) unsigned char tma_smem[];  // the tensor copy's destination
  constexpr int K = LR1 + LR2;
  uint64_t *bar = reinterpret_cast<uint64_t *>(tma_smem + tma_bar_off<F, LR1, LR2, C>());
  if (threadIdx.x == 0) {
    const uint32_t chunk = blockIdx.x % g.chunks_per_row, rest = blockIdx.x / g.chunks_per_row;
    const uint32_t grp = rest % g.groups, blk = rest / g.groups;
    const uint32_t i_low = grp & ((1u << g.lo) - 1u);
    const uint32_t high = blk * (g.groups >> g.lo) + (grp >> g.lo);  // row bits above the pass, transform
    mbar_init(bar, 1);
    mbar_expect_tx(bar, (uint32_t)((C << K) * sizeof(typename F::T)));
    tma_load_5d(tma_smem, &map, bar, (int)(chunk * C), (int)i_low, 0, 0, (int)high);
  }
  __syncthreads();  // the barrier is initialised before anyone waits on it
  ntt_pass_tile<F, LR1, LR2, C, false, true>(in, out, g, tw, post_scale, st, blockIdx.x, tma_smem, bar,
                                             &g_tma_wait_errors);
}

// Tile loads of the passes and the fused middle: 1 = one tensor copy per tile (the
// default; measured 0.6-12.5 % faster than register loads on BabyBear and Goldilocks LDEs
// of 2^18..2^22 rows), 0 = coalesced loads into registers.  Set by zkb_set_ntt_tile_loads or
// ZKB_NTT_TMA=0/1.
std::atomic<int> &ntt_tile_loads() {
  static std::atomic<int> mode{[] {
    const char *v = getenv("ZKB_NTT_TMA");
    return v && *v == '0' ? 0 : 1;
  }()};
  return mode;
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return (EncodeTiledFn)p;
  }();
  return fn;
}

// Tensor map of one column segment (`cols` columns of `es`-byte elements from `base`, row
// stride g.width) for the tiles of a K-bit pass at bits [g.lo, g.lo + K): dimensions
// (column, row bits below the pass, the pass's bits split 8 + rest, the bits above with
// the transform index), box C columns x 2^K rows.  The caller has checked that the row
// stride, the base and C * es are multiples of 16 bytes (every copy starts at a column
// that is a multiple of C).
static int pass_tensor_map(CUtensorMap *m, const void *base, size_t es, const PassGeom &g, uint32_t cols, int K,
                           uint64_t n_blocks, uint32_t C) {
  const EncodeTiledFn fn = encode_tiled();
  ZKB_REQUIRE(fn != nullptr, "cuTensorMapEncodeTiled is not available");
  const int K1 = K < 8 ? K : 8, K2 = K - K1;
  const uint64_t row = (uint64_t)g.width * es;
  const cuuint64_t dims[5] = {cols, 1ull << g.lo, 1ull << K1, 1ull << K2, (1ull << (g.L - g.lo - K)) * n_blocks};
  const cuuint64_t strides[4] = {row, row << g.lo, row << (g.lo + K1), row << (g.lo + K)};
  const cuuint32_t box[5] = {C, 1, 1u << K1, 1u << K2, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult r = fn(m, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_UINT64, 5, (void *)base,
                        dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  ZKB_REQUIRE(r == CUDA_SUCCESS, "tensor map of an NTT pass refused (error %d)", (int)r);
  return ZKB_OK;
}

// Whether the tiles of a K-bit pass at bits [lo, lo + K) of `n_blocks` transforms of 2^L
// rows can come by tensor copy: the mode is on, C columns and the row stride are multiples of
// 16 bytes, the base is 16-byte aligned, and the tensor map's limits hold (strides below
// 2^40 bytes, dimensions up to 2^32).  Otherwise the tile keeps its register loads.
static bool tma_tiles(const void *base, size_t es, uint32_t width, uint32_t C, int L, int lo, int K, uint64_t n_blocks,
                      uint32_t cols) {
  if (!cols || ntt_tile_loads().load() != 1 || C * es < 16 || (width * es) % 16 != 0 || ((uintptr_t)base & 15) != 0)
    return false;
  const uint64_t row = (uint64_t)width * es;
  if (L - lo - K < 0 || lo + K > 40 || (row << (lo + K)) >= (1ull << 40) || (row >> (40 - lo - K)) != 0) return false;
  return ((1ull << (L - lo - K)) * n_blocks) <= (1ull << 32);
}

template <class F, int LR1, int LR2, int C>
static int launch_pass_tma_c(const typename F::T *src, typename F::T *out, const PassGeom &g, uint32_t cols,
                             uint64_t n_blocks, uint64_t ctas, const typename F::T *tw, typename F::T scale,
                             const SmallTw<F> &st, cudaStream_t s) {
  constexpr unsigned threads = C << LR2;
  const size_t smem = tma_bar_off<F, LR1, LR2, C>() + 16;
  CUtensorMap map;
  ZKB_TRY(pass_tensor_map(&map, src, sizeof(typename F::T), g, cols, LR1 + LR2, n_blocks, C));
  ZKB_CHECK_CUDA(cudaFuncSetAttribute(ntt_pass_tma_kernel<F, LR1, LR2, C>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  ZKB_LAUNCH("ntt_pass_tma", s, ntt_pass_tma_kernel<F, LR1, LR2, C><<<(unsigned)ctas, threads, smem, s>>>(src, out, g, tw, scale, st, map));
  return ZKB_OK;
}

// Column segments of a `width`-column matrix: the widest chunk (at most cmax columns per
// CTA) for the bulk, then narrower chunks (8, 4, 1) for what is left, each launched on
// offset pointers with the full row stride.  Every width keeps coalesced rows for all
// but at most cmax - 1 columns.
struct ColSeg {
  uint32_t col0, cols, C;
};
static std::vector<ColSeg> col_segments(uint32_t width, uint32_t cmax) {
  std::vector<ColSeg> v;
  uint32_t c0 = 0;
  for (uint32_t C : {16u, 8u, 4u, 1u}) {
    if (C > cmax) continue;
    const uint32_t n = (width - c0) / C;
    if (n) {
      v.push_back(ColSeg{c0, n * C, C});
      c0 += n * C;
    }
  }
  return v;
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
    st.w[e] = acc;
    if constexpr (sizeof(typename F::T) == 4)
      st.q[e] = BabyBear::shoup_quotient(acc);
    else
      st.q[e] = 0;
    acc = F::mul_host(acc, w);
  }
  return st;
}

template <class F, int LR1, int LR2, int C>
static int launch_pass_c(const typename F::T *src, typename F::T *out, const PassGeom &g, uint64_t ctas,
                         const typename F::T *tw, typename F::T scale, const SmallTw<F> &st,
                         cudaStream_t s) {
  using T = typename F::T;
  constexpr unsigned threads = C << LR2;
  const size_t smem = pass_tile_smem<F, LR1, LR2, C>();
  ZKB_CHECK_CUDA(cudaFuncSetAttribute(ntt_pass_kernel<F, LR1, LR2, C>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  ZKB_LAUNCH("ntt_pass", s, ntt_pass_kernel<F, LR1, LR2, C><<<(unsigned)ctas, threads, smem, s>>>(src, out, g, tw, scale, st));
  return ZKB_OK;
}

template <class F, int LR1, int LR2>
static int launch_pass(const typename F::T *src, typename F::T *out, const PassGeom &g, uint64_t ctas,
                       const typename F::T *tw, typename F::T scale, const SmallTw<F> &st,
                       uint32_t C, cudaStream_t s, uint32_t cols = 0, uint64_t n_blocks = 0) {
  // tensor-copy tile loads where every copy's start and the row stride are 16-byte aligned
  if (tma_tiles(src, sizeof(typename F::T), g.width, C, g.L, g.lo, LR1 + LR2, n_blocks, cols)) {
    switch (C) {
      case 16:
        if constexpr (sizeof(typename F::T) == 4) return launch_pass_tma_c<F, LR1, LR2, 16>(src, out, g, cols, n_blocks, ctas, tw, scale, st, s);
        break;
      case 8: return launch_pass_tma_c<F, LR1, LR2, 8>(src, out, g, cols, n_blocks, ctas, tw, scale, st, s);
      case 4: return launch_pass_tma_c<F, LR1, LR2, 4>(src, out, g, cols, n_blocks, ctas, tw, scale, st, s);
      default: break;
    }
  }
  switch (C) {
    case 16:
      if constexpr (sizeof(typename F::T) == 4) return launch_pass_c<F, LR1, LR2, 16>(src, out, g, ctas, tw, scale, st, s);
      break;
    case 8: return launch_pass_c<F, LR1, LR2, 8>(src, out, g, ctas, tw, scale, st, s);
    case 4: return launch_pass_c<F, LR1, LR2, 4>(src, out, g, ctas, tw, scale, st, s);
    case 1: return launch_pass_c<F, LR1, LR2, 1>(src, out, g, ctas, tw, scale, st, s);
    default: break;
  }
  set_error("internal: NTT column chunk %u", C);
  return ZKB_ERR_INTERNAL;
}

// Largest pass of the default plans (the kernels exist up to 11 bits for BabyBear and 10
// for Goldilocks, which explicit tuning can still ask for).  Measured on B200 over
// heights 2^12..2^24: BabyBear is at or near its best with passes of at most 10 bits
// (an 11-bit pass holds 64 values per thread and runs at lower occupancy), Goldilocks
// with at most 7 (its 8-byte tiles fill shared memory twice as fast).
template <class F>
static constexpr int pass_kmax() {
  return sizeof(typename F::T) == 4 ? 10 : 7;
}

// Runs the passes `ks` (bit counts, top first) starting at index bit hi_start, over
// `width` columns of a matrix whose rows are `stride` elements apart (0: width).
template <class F>
static int run_plan(const typename F::T *in, typename F::T *out, int L, uint32_t width,
                    uint64_t n_blocks, const typename F::T *tw, bool inverse,
                    typename F::T last_scale, const std::vector<int> &ks, int hi_start,
                    cudaStream_t s, uint32_t cmax = 0, uint32_t stride = 0) {
  using T = typename F::T;
  if (cmax == 0) cmax = sizeof(T) == 4 ? 16 : 8;
  if (stride == 0) stride = width;
  const std::vector<ColSeg> segs = col_segments(width, cmax);
  // the register DIFs use w_64 of the same direction as the table `tw`
  const SmallTw<F> st = small_twiddles<F>(inverse);
  int hi = hi_start;
  const T *src = in;
  for (size_t pi = 0; pi < ks.size(); pi++) {
    const int K = ks[pi];
    PassGeom g;
    g.L = L;
    g.lo = hi - K;
    g.width = stride;
    g.groups = 1u << (L - K);
    g.block_stride = ((uint64_t)stride) << L;
    g.twist = g.lo > 0;
    if (((uint64_t)stride << L) * n_blocks >= (1ull << 40)) {
      set_error("NTT launch too large");
      return ZKB_ERR_UNSUPPORTED;
    }
    const T scale = (pi + 1 == ks.size()) ? last_scale : (T)0;
    int rc = ZKB_OK;
    for (const ColSeg &sg : segs) {
      const uint32_t C = sg.C;
      const T *sp = src + sg.col0;
      T *op = out + sg.col0;
      g.chunks_per_row = sg.cols / C;
      const uint64_t ctas = (uint64_t)g.chunks_per_row * g.groups * n_blocks;
      if (ctas >= (1ull << 31)) {
        set_error("NTT launch too large");
        return ZKB_ERR_UNSUPPORTED;
      }
      switch (K) {
        case 1: rc = launch_pass<F, 1, 0>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 2: rc = launch_pass<F, 1, 1>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 3: rc = launch_pass<F, 2, 1>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 4: rc = launch_pass<F, 2, 2>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 5: rc = launch_pass<F, 3, 2>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 6: rc = launch_pass<F, 3, 3>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 7: rc = launch_pass<F, 4, 3>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 8: rc = launch_pass<F, 4, 4>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 9: rc = launch_pass<F, 5, 4>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 10: rc = launch_pass<F, 5, 5>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks); break;
        case 11:
          if constexpr (sizeof(T) == 4) {
            rc = launch_pass<F, 6, 5>(sp, op, g, ctas, tw, scale, st, C, s, sg.cols, n_blocks);
            break;
          }
          [[fallthrough]];
        default:
          set_error("internal: NTT pass of %d bits", K);
          return ZKB_ERR_INTERNAL;
      }
      ZKB_TRY(rc);
    }
    ZKB_TRY(rc);
    src = out;
    hi = g.lo;
  }
  return ZKB_OK;
}

template <class F>
static int run_passes(const typename F::T *in, typename F::T *out, int L, uint32_t width,
                      uint64_t n_blocks, const typename F::T *tw, bool inverse,
                      typename F::T last_scale, cudaStream_t s) {
  return run_plan<F>(in, out, L, width, n_blocks, tw, inverse, last_scale,
                     plan_passes(L, pass_kmax<F>()), L, s);
}

// --------------------------------------------------------- fused LDE middle
// (geometry and tile code: ntt_tile.cuh)
template <class F, int LR1, int LR2, int C>
__global__ void __launch_bounds__(C << LR2)
    lde_fused_kernel(const typename F::T *in, typename F::T *out, const FusedGeom g,
                     const typename F::T *__restrict__ itw, const typename F::T *__restrict__ ftw,
                     const typename F::T *__restrict__ ctab_t, const typename F::T *__restrict__ ftw_t,
                     const __grid_constant__ SmallTw<F> ist, const __grid_constant__ SmallTw<F> fst) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  lde_fused_tile<F, LR1, LR2, C, false>(in, out, g, itw, ftw, ctab_t, ftw_t, ist, fst, blockIdx.x, smem_raw);
}

// The fused middle with block B's rows brought in by one tensor copy (as the passes).
template <class F, int LR1, int LR2, int C>
constexpr size_t fused_bar_off() {
  return (fused_tile_smem<F, LR1, LR2, C>() + 15) & ~(size_t)15;
}

template <class F, int LR1, int LR2, int C>
__global__ void __launch_bounds__(C << LR2)
    lde_fused_tma_kernel(const typename F::T *in, typename F::T *out, const FusedGeom g,
                         const typename F::T *__restrict__ itw, const typename F::T *__restrict__ ftw,
                         const typename F::T *__restrict__ ctab_t, const typename F::T *__restrict__ ftw_t,
                         const __grid_constant__ SmallTw<F> ist, const __grid_constant__ SmallTw<F> fst,
                         const __grid_constant__ CUtensorMap map) {
  extern __shared__ __align__(128) unsigned char tma_smem[];
  constexpr int K = LR1 + LR2;
  uint64_t *bar = reinterpret_cast<uint64_t *>(tma_smem + fused_bar_off<F, LR1, LR2, C>());
  if (threadIdx.x == 0) {
    const uint32_t chunk = blockIdx.x % g.chunks_per_row, B = blockIdx.x / g.chunks_per_row;
    mbar_init(bar, 1);
    mbar_expect_tx(bar, (uint32_t)((C << K) * sizeof(typename F::T)));
    tma_load_5d(tma_smem, &map, bar, (int)(chunk * C), 0, 0, 0, (int)B);
  }
  __syncthreads();  // the barrier is initialised before anyone waits on it
  lde_fused_tile<F, LR1, LR2, C, false, true>(in, out, g, itw, ftw, ctab_t, ftw_t, ist, fst, blockIdx.x, tma_smem,
                                              bar, &g_tma_wait_errors);
}

template <class F, int LR1, int LR2, int C>
static int launch_fused_c(const typename F::T *in, typename F::T *out, const FusedGeom &g,
                          const typename F::T *itw, const typename F::T *ftw, const typename F::T *ctab,
                          const typename F::T *ftw_t, cudaStream_t s, uint32_t cols) {
  using T = typename F::T;
  constexpr unsigned threads = C << LR2;
  const uint64_t ctas0 = (uint64_t)g.chunks_per_row * g.blocks;
  if (tma_tiles(in, sizeof(T), g.width, C, g.L, 0, LR1 + LR2, 1, cols)) {
    // block B's rows as the tile of a pass at bits [0, K) of one transform
    PassGeom pg;
    pg.L = g.L;
    pg.lo = 0;
    pg.width = g.width;
    CUtensorMap map;
    ZKB_TRY(pass_tensor_map(&map, in, sizeof(T), pg, cols, LR1 + LR2, 1, C));
    const size_t smem = fused_bar_off<F, LR1, LR2, C>() + 16;
    ZKB_CHECK_CUDA(cudaFuncSetAttribute(lde_fused_tma_kernel<F, LR1, LR2, C>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    const SmallTw<F> ist = small_twiddles<F>(true), fst = small_twiddles<F>(false);
    ZKB_LAUNCH("lde_fused_tma", s, lde_fused_tma_kernel<F, LR1, LR2, C><<<(unsigned)ctas0, threads, smem, s>>>(in, out, g, itw, ftw, ctab, ftw_t, ist, fst, map));
    return ZKB_OK;
  }
  const size_t smem = fused_tile_smem<F, LR1, LR2, C>();
  ZKB_CHECK_CUDA(cudaFuncSetAttribute(lde_fused_kernel<F, LR1, LR2, C>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  const uint64_t ctas = (uint64_t)g.chunks_per_row * g.blocks;
  const SmallTw<F> ist = small_twiddles<F>(true), fst = small_twiddles<F>(false);
  ZKB_LAUNCH("lde_fused", s, lde_fused_kernel<F, LR1, LR2, C><<<(unsigned)ctas, threads, smem, s>>>(in, out, g, itw, ftw, ctab, ftw_t, ist, fst));
  return ZKB_OK;
}

// Column chunk of the fused kernel: it holds 2 x R1 values per thread, so BabyBear uses
// 8 columns (256 threads, up to 255 registers) where the plain passes use 16.
template <class F, int LR1, int LR2>
static int launch_fused(const typename F::T *in, typename F::T *out, const FusedGeom &g,
                        const typename F::T *itw, const typename F::T *ftw, const typename F::T *ctab,
                        const typename F::T *ftw_t, uint32_t C, cudaStream_t s, uint32_t cols) {
  switch (C) {
    case 8: return launch_fused_c<F, LR1, LR2, 8>(in, out, g, itw, ftw, ctab, ftw_t, s, cols);
    case 4: return launch_fused_c<F, LR1, LR2, 4>(in, out, g, itw, ftw, ctab, ftw_t, s, cols);
    case 1: return launch_fused_c<F, LR1, LR2, 1>(in, out, g, itw, ftw, ctab, ftw_t, s, cols);
    default: break;
  }
  set_error("internal: fused LDE column chunk %u", C);
  return ZKB_ERR_INTERNAL;
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
static int launch_fused_k(int K, const typename F::T *in, typename F::T *out, const FusedGeom &g,
                          const typename F::T *itw, const typename F::T *ftw, const typename F::T *ctab,
                          const typename F::T *ftw_t, uint32_t C, cudaStream_t s, uint32_t cols) {
  switch (K) {
    case 1: return launch_fused<F, 1, 0>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 2: return launch_fused<F, 1, 1>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 3: return launch_fused<F, 2, 1>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 4: return launch_fused<F, 2, 2>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 5: return launch_fused<F, 3, 2>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 6: return launch_fused<F, 3, 3>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 7: return launch_fused<F, 4, 3>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 8: return launch_fused<F, 4, 4>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 9: return launch_fused<F, 5, 4>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 10: return launch_fused<F, 5, 5>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
    case 11:
      if constexpr (sizeof(typename F::T) == 4) return launch_fused<F, 6, 5>(in, out, g, itw, ftw, ctab, ftw_t, C, s, cols);
      [[fallthrough]];
    default:
      set_error("internal: fused LDE pass of %d bits", K);
      return ZKB_ERR_INTERNAL;
  }
}

// Coset LDE, rows bit-reversed (the PCS order):
//   inverse passes over all but the lowest K bits (trace -> coefficient scratch),
//   lde_fused_kernel (last inverse pass + coset twists + first forward pass),
//   the remaining forward passes in place on the 2^log_b coset blocks,
// with the forward plan the mirror of the inverse one so both meet at K bits.
int lde_tune_check(int field, uint32_t width, const LdeTune &t) {
  const int kmax = field == FIELD_BABYBEAR ? 11 : 10;
  const uint32_t cmax = field == FIELD_BABYBEAR ? 16 : 8;
  ZKB_REQUIRE(t.kmax >= 0 && t.kmax <= kmax, "LDE tuning: pass size %d out of range", t.kmax);
  (void)width;  // widths that are not a multiple of the chunk take narrower chunks for the rest
  ZKB_REQUIRE(t.c_pass == 0 || ((t.c_pass == 1 || t.c_pass == 4 || t.c_pass == 8 || t.c_pass == 16) &&
                                t.c_pass <= cmax),
              "LDE tuning: pass column chunk %u not in {1, 4, 8, 16} (at most %u)", t.c_pass, cmax);
  ZKB_REQUIRE(t.c_fused == 0 || t.c_fused == 1 || t.c_fused == 4 || t.c_fused == 8,
              "LDE tuning: fused column chunk %u not in {1, 4, 8}", t.c_fused);
  return ZKB_OK;
}

// Coset LDE, rows bit-reversed (the PCS order):
//   inverse passes over all but the lowest K bits (trace -> coefficient scratch),
//   lde_fused_kernel (last inverse pass + coset twists + first forward pass),
//   the remaining forward passes in place on the 2^log_b coset blocks,
// with the forward plan the mirror of the inverse one so both meet at K bits.
// `tune` overrides the pass size and column chunks (zero fields keep the defaults);
// `coef_scratch` (2^log_h x width elements), when given, replaces the scratch
// allocation, so that with bitrev set the call allocates nothing.
template <class F>
int ntt_lde_dev(const typename F::T *d_trace, int log_h, uint32_t width, int log_b,
                typename F::T shift, bool bitrev, typename F::T *d_out, cudaStream_t s,
                const LdeTune *tune, typename F::T *coef_scratch, uint32_t stride) {
  using T = typename F::T;
  if (width == 0) return ZKB_OK;
  if (log_h + log_b > F::TWO_ADICITY) {
    set_error("LDE size 2^%d exceeds the two-adicity of the field", log_h + log_b);
    return ZKB_ERR_INVALID;
  }
  if (stride == 0) stride = width;
  ZKB_REQUIRE(stride == width || (stride > width && bitrev && log_h > 0 && coef_scratch != nullptr),
              "internal: an LDE of some columns of a wider matrix needs bit-reversed rows, a height above 1 "
              "and a coefficient scratch of the same stride");
  LdeTune tn;
  if (tune) {
    ZKB_TRY(lde_tune_check(field_id<F>(), width, *tune));
    tn = *tune;
  }
  const int kmax = tn.kmax ? tn.kmax : pass_kmax<F>();
  const uint64_t n = 1ull << log_h;
  const T *ctab;
  ZKB_TRY(get_coset_table<F>(log_h, log_b, shift, &ctab, s));
  if (log_h == 0) {
    // a single row: every evaluation is the constant coefficient
    ZKB_LAUNCH("lde_expand", s, lde_expand_kernel<F><<<grid_for(width, 256), 256, 0, s>>>(d_trace, d_out, 0, log_b, width, ctab));
  } else {
    const T *itw, *ftw;
    ZKB_TRY(get_twiddles<F>(log_h, true, &itw, s));
    ZKB_TRY(get_twiddles<F>(log_h, false, &ftw, s));
    const std::vector<int> ks = plan_passes(log_h, kmax);
    const int Kf = ks.back();
    ScratchBuf coef;
    const T *src = d_trace;
    if (ks.size() > 1) {
      T *cs = coef_scratch;
      if (!cs) {
        ZKB_TRY(coef.alloc(n * width * sizeof(T), s));
        cs = coef.as<T>();
      }
      std::vector<int> head(ks.begin(), ks.end() - 1);
      ZKB_TRY(run_plan<F>(d_trace, cs, log_h, width, 1, itw, true, (T)0, head, log_h, s, tn.c_pass, stride));
      src = cs;
    }
    FusedGeom g;
    g.L = log_h;
    g.width = stride;
    g.blocks = 1u << (log_h - Kf);
    g.log_b = log_b;
    g.n = n;
    const T *ctab_t, *ftw_t;
    ZKB_TRY(get_fused_tables<F>(log_h, log_b, shift, Kf, ctab, ftw, &ctab_t, &ftw_t, s));
    for (const ColSeg &sg : col_segments(width, tn.c_fused ? tn.c_fused : 8)) {
      g.chunks_per_row = sg.cols / sg.C;
      if ((uint64_t)g.chunks_per_row * g.blocks >= (1ull << 31)) {
        set_error("LDE launch too large");
        return ZKB_ERR_UNSUPPORTED;
      }
      ZKB_TRY(launch_fused_k<F>(Kf, src + sg.col0, d_out + sg.col0, g, itw, ftw, ctab_t, ftw_t, sg.C, s, sg.cols));
    }
    std::vector<int> tail(ks.rbegin() + 1, ks.rend());
    if (!tail.empty())
      ZKB_TRY(run_plan<F>(d_out, d_out, log_h, width, 1ull << log_b, ftw, false, (T)0, tail,
                          log_h - Kf, s, tn.c_pass, stride));
  }
  if (!bitrev) {
    const int LN = log_h + log_b;
    const uint64_t total = (n << log_b) * width;
    ScratchBuf tmp;
    ZKB_TRY(tmp.alloc(total * sizeof(T), s));
    ZKB_LAUNCH("bitrev_rows", s, bitrev_rows_kernel<F><<<grid_for(total, 256), 256, 0, s>>>(d_out, tmp.as<T>(), LN, width, total));
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

void small_twiddles_bb(bool inverse, SmallTw<BabyBear> *out) { *out = small_twiddles<BabyBear>(inverse); }

int lde_plan_babybear(int log_h, int log_b, int kmax, LdePlanBB *out, cudaStream_t s) {
  ZKB_REQUIRE(log_h >= 1 && log_h + log_b <= BabyBear::TWO_ADICITY, "LDE of 2^%d rows x2^%d", log_h, log_b);
  out->ks = plan_passes(log_h, kmax);
  const uint32_t *ctab;
  ZKB_TRY(get_coset_table<BabyBear>(log_h, log_b, BabyBear::GENERATOR, &ctab, s));
  ZKB_TRY(get_twiddles<BabyBear>(log_h, true, &out->itw, s));
  ZKB_TRY(get_twiddles<BabyBear>(log_h, false, &out->ftw, s));
  return get_fused_tables<BabyBear>(log_h, log_b, BabyBear::GENERATOR, out->ks.back(), ctab, out->ftw,
                                    &out->ctab_t, &out->ftw_t, s);
}

template int get_twiddles<BabyBear>(int, bool, const uint32_t **, cudaStream_t);
template int get_twiddles<Goldilocks>(int, bool, const uint64_t **, cudaStream_t);
template int ntt_dft_dev<BabyBear>(uint32_t *, int, uint32_t, bool, cudaStream_t);
template int ntt_dft_dev<Goldilocks>(uint64_t *, int, uint32_t, bool, cudaStream_t);
template int ntt_lde_dev<BabyBear>(const uint32_t *, int, uint32_t, int, uint32_t, bool, uint32_t *,
                                   cudaStream_t, const LdeTune *, uint32_t *, uint32_t);
template int ntt_lde_dev<Goldilocks>(const uint64_t *, int, uint32_t, int, uint64_t, bool,
                                     uint64_t *, cudaStream_t, const LdeTune *, uint64_t *, uint32_t);

void set_ntt_tile_loads(int mode) { ntt_tile_loads().store(mode); }
int ntt_tile_loads_mode() { return ntt_tile_loads().load(); }

int ntt_tma_wait_errors(uint32_t *count) {
  uint32_t v = 0;
  ZKB_CHECK_CUDA(cudaMemcpyFromSymbol(&v, g_tma_wait_errors, sizeof v));
  const uint32_t zero = 0;
  ZKB_CHECK_CUDA(cudaMemcpyToSymbol(g_tma_wait_errors, &zero, sizeof zero));
  *count = v;
  return ZKB_OK;
}

}  // namespace zkb
