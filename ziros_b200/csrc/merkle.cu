// merkle.cu — Poseidon2 MMCS: leaf sponge hashing, 2-to-1 compression, tree layers.
//
// Semantics follow p3 MerkleTree::new as vendored in
// vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:84-151 (first_digest_layer :202-266,
// compress_and_inject :272-350, compress :359-403) with
//   leaf  = PaddingFreeSponge<Perm, W, 8, OUT> over the concatenated rows of the
//           tallest matrices (overwrite-mode absorption, partial last chunk keeps
//           the old lanes, zkf-backends/src/wrapping/poseidon2_goldilocks.rs:392-415);
//   node  = TruncatedPermutation<Perm, 2, OUT, W> (poseidon2_goldilocks.rs:373-390);
//   layer lengths padded to even with zero digests except at the root; shorter
//   matrices injected as compress(compress(l, r), hash(rows)).
// Unlike the reference's Metal path (zkf-metal/src/merkle.rs:82-90), which falls back
// to the CPU for rows wider than 8 elements, every width is hashed on the device.
#include <algorithm>
#include <type_traits>
#include <numeric>

#include "common.cuh"
#include "engine.cuh"
#include "poseidon2.cuh"

namespace zkb {

constexpr int MAX_GROUP_MATS = 16;

struct MatList {
  const void *ptr[MAX_GROUP_MATS];
  uint64_t width[MAX_GROUP_MATS];
  uint64_t col_start[MAX_GROUP_MATS + 1];
  int n;
};

template <int W>
__host__ __device__ constexpr int p2_out() {
  return W == 16 ? 8 : 4;
}

template <class F>
__device__ __forceinline__ typename F::T fetch_col(const MatList &ml, uint64_t row, uint64_t col) {
  int m = 0;
  while (m + 1 < ml.n && col >= ml.col_start[m + 1]) m++;
  const typename F::T *base = (const typename F::T *)ml.ptr[m];
  return base[row * ml.width[m] + (col - ml.col_start[m])];
}

// Leaf digests: PaddingFreeSponge over the concatenated row of the matrices in ml.
// One permutation call site per kernel (keeps the code within the instruction cache);
// a partial last chunk overwrites only its own lanes.
template <class F, int W>
__global__ void __launch_bounds__(128)
    hash_rows_kernel(const MatList ml, uint64_t height, typename F::T *__restrict__ digests,
                     const __grid_constant__ P2Params<F, W> p) {
  using T = typename F::T;
  using D = Dom<F>;
  constexpr int OUT = p2_out<W>();
  const uint64_t total = ml.col_start[ml.n];
  for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < height;
       row += (uint64_t)gridDim.x * blockDim.x) {
    T s[W];
#pragma unroll
    for (int i = 0; i < W; i++) s[i] = 0;
    const T *rp = (const T *)ml.ptr[0] + row * ml.width[0];
    for (uint64_t c = 0; c < total; c += 8) {
      if (ml.n == 1) {
#pragma unroll
        for (int i = 0; i < 8; i++)
          if (c + i < total) s[i] = D::enter(rp[c + i]);
      } else {
#pragma unroll
        for (int i = 0; i < 8; i++)
          if (c + i < total) s[i] = D::enter(fetch_col<F>(ml, row, c + i));
      }
      p2_permute<F, W>(s, p);
    }
#pragma unroll
    for (int i = 0; i < OUT; i++) digests[row * OUT + i] = D::leave(s[i]);
  }
}

// The leaf sponge of one BabyBear matrix with the alpha-reduction of each row fused in:
// while the row streams through the sponge, out[row] accumulates sum_j alpha^j * row[j]
// (four Montgomery products per element, 64-bit sums reduced once; the powers are
// encoded alpha^j * 2^64 so one reduction gives the canonical sum).
__global__ void __launch_bounds__(128)
    hash_rows_combine_kernel(const uint32_t *__restrict__ mat, uint64_t width, uint64_t height,
                             uint32_t *__restrict__ digests, const __grid_constant__ P2Params<BabyBear, 16> p,
                             const uint4 *__restrict__ apow, uint4 *__restrict__ comb) {
  using D = Dom<BabyBear>;
  using B = BabyBear;
  for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < height;
       row += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s[16];
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = 0;
    // Two columns per reduction: v0*w0 + v1*w1 < 2p^2 < p*2^32 is one Montgomery
    // reduction's input, so a pair costs two wide multiply-adds and one reduction.
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    const uint32_t *rp = mat + row * width;
    for (uint64_t c = 0; c < width; c += 8) {
#pragma unroll
      for (int i = 0; i < 8; i += 2) {
        if (c + i < width) {
          const uint32_t v0 = rp[c + i];
          const uint4 w0 = apow[c + i];
          s[i] = D::enter(v0);
          uint32_t v1 = 0;
          uint4 w1 = make_uint4(0, 0, 0, 0);
          if (c + i + 1 < width) {
            v1 = rp[c + i + 1];
            w1 = apow[c + i + 1];
            s[i + 1] = D::enter(v1);
          }
          a0 += B::mont_lazy_sum(v0, w0.x, v1, w1.x);
          a1 += B::mont_lazy_sum(v0, w0.y, v1, w1.y);
          a2 += B::mont_lazy_sum(v0, w0.z, v1, w1.z);
          a3 += B::mont_lazy_sum(v0, w0.w, v1, w1.w);
        }
      }
      p2_permute<BabyBear, 16>(s, p);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) digests[row * 8 + i] = D::leave(s[i]);
    comb[row] = make_uint4(B::mont_reduce(a0), B::mont_reduce(a1), B::mont_reduce(a2), B::mont_reduce(a3));
  }
}

// The same sponge over columns [c0, c0 + ncols) of the rows only (row stride `stride`), for a
// matrix that arrives a slab of columns at a time: the sponge state comes from `carry`
// (16 words per row, internal domain; none on the first slab) and goes back there, or on
// the last slab the digest goes to `digests`.  c0 is a multiple of 8 (slabs hold whole
// absorbed chunks; only the last slab may end in a partial one), so the chunks and
// permutations are exactly the full row's.  With apow, the rows' alpha-reduction over
// these columns is written (first slab) or added (mod p) to comb: the sum of the slabs'
// reductions is the whole row's.
__global__ void __launch_bounds__(128)
    hash_rows_slab_kernel(const uint32_t *__restrict__ mat, uint64_t stride, uint64_t c0, uint64_t ncols,
                          uint64_t height, uint32_t *__restrict__ carry, int first, int last,
                          uint32_t *__restrict__ digests, const __grid_constant__ P2Params<BabyBear, 16> p,
                          const uint4 *__restrict__ apow, uint4 *__restrict__ comb) {
  using D = Dom<BabyBear>;
  using B = BabyBear;
  for (uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; row < height;
       row += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s[16];
    if (first) {
#pragma unroll
      for (int i = 0; i < 16; i++) s[i] = 0;
    } else {
      const uint4 *cp = reinterpret_cast<const uint4 *>(carry + row * 16);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint4 v = cp[q];
        s[4 * q] = v.x;
        s[4 * q + 1] = v.y;
        s[4 * q + 2] = v.z;
        s[4 * q + 3] = v.w;
      }
    }
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    const uint32_t *rp = mat + row * stride + c0;
    const uint4 *ap = apow ? apow + c0 : nullptr;
    for (uint64_t c = 0; c < ncols; c += 8) {
#pragma unroll
      for (int i = 0; i < 8; i += 2) {
        if (c + i < ncols) {
          const uint32_t v0 = rp[c + i];
          s[i] = D::enter(v0);
          uint32_t v1 = 0;
          if (c + i + 1 < ncols) {
            v1 = rp[c + i + 1];
            s[i + 1] = D::enter(v1);
          }
          if (ap) {
            const uint4 w0 = ap[c + i];
            const uint4 w1 = c + i + 1 < ncols ? ap[c + i + 1] : make_uint4(0, 0, 0, 0);
            a0 += B::mont_lazy_sum(v0, w0.x, v1, w1.x);
            a1 += B::mont_lazy_sum(v0, w0.y, v1, w1.y);
            a2 += B::mont_lazy_sum(v0, w0.z, v1, w1.z);
            a3 += B::mont_lazy_sum(v0, w0.w, v1, w1.w);
          }
        }
      }
      p2_permute<BabyBear, 16>(s, p);
    }
    if (last) {
#pragma unroll
      for (int i = 0; i < 8; i++) digests[row * 8 + i] = D::leave(s[i]);
    } else {
      uint4 *cp = reinterpret_cast<uint4 *>(carry + row * 16);
#pragma unroll
      for (int q = 0; q < 4; q++) cp[q] = make_uint4(s[4 * q], s[4 * q + 1], s[4 * q + 2], s[4 * q + 3]);
    }
    if (ap) {
      uint4 r = make_uint4(B::mont_reduce(a0), B::mont_reduce(a1), B::mont_reduce(a2), B::mont_reduce(a3));
      if (!first) {
        const uint4 o = comb[row];
        r = make_uint4(B::add(o.x, r.x), B::add(o.y, r.y), B::add(o.z, r.z), B::add(o.w, r.w));
      }
      comb[row] = r;
    }
  }
}

// next[i] = compress(prev[2i], prev[2i+1]); with `inj` (digests of the rows injected at
// this layer, inj_h of them) next[i] = compress(that, i < inj_h ? inj[i] : 0).
template <class F, int W>
__global__ void __launch_bounds__(128)
    compress_kernel(const typename F::T *__restrict__ prev, typename F::T *__restrict__ next,
                    uint64_t n_out, const typename F::T *__restrict__ inj, uint64_t inj_h,
                    const __grid_constant__ P2Params<F, W> p) {
  using T = typename F::T;
  using D = Dom<F>;
  constexpr int OUT = p2_out<W>();
  const int rounds = inj ? 2 : 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x) {
    T s[W];
#pragma unroll
    for (int k = 0; k < OUT; k++) {
      s[k] = D::enter(prev[(2 * i) * OUT + k]);
      s[OUT + k] = D::enter(prev[(2 * i + 1) * OUT + k]);
    }
    for (int r = 0; r < rounds; r++) {
      if (r == 1) {
#pragma unroll
        for (int k = 0; k < OUT; k++) s[OUT + k] = i < inj_h ? D::enter(inj[i * OUT + k]) : (T)0;
      }
#pragma unroll
      for (int k = 2 * OUT; k < W; k++) s[k] = 0;
      p2_permute<F, W>(s, p);
    }
#pragma unroll
    for (int k = 0; k < OUT; k++) next[i * OUT + k] = D::leave(s[k]);
  }
}

DeviceTree::~DeviceTree() {
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  if (d_layers && !borrowed) dev_free(d_layers, stream);
  for (void *p : owned) dev_free(p, stream);
  cudaSetDevice(prev);
}

static uint64_t next_pow2_u64(uint64_t x) { return ceil_pow2(x); }

static int log2_ceil(uint64_t x) {
  int l = 0;
  while ((1ull << l) < x) l++;
  return l;
}

template <class F, int W>
static int build_tree_impl(const HasherSpec &h, const std::vector<TreeMatrix> &mats,
                           DeviceTree *t, cudaStream_t s, bool fri_layer, const LeafCombine *comb,
                           const LeafFill *fill) {
  const char *leaf_name = fri_layer ? "fri_leaf_hash" : "merkle_leaf_hash";
  const char *comp_name = fri_layer ? "fri_compress" : "merkle_compress";
  using T = typename F::T;
  constexpr int OUT = p2_out<W>();
  P2Params<F, W> p;
  if (!build_p2_params<F, W>(h, &p)) {
    set_error("invalid Poseidon2 parameters");
    return ZKB_ERR_INVALID;
  }
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));

  const size_t nm = mats.size();
  std::vector<size_t> ord(nm);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](size_t a, size_t b) { return mats[a].height > mats[b].height; });
  const uint64_t max_h = mats[ord[0]].height;
  ZKB_REQUIRE(max_h > 0, "matrix height 0 not supported");
  const int log_max = log2_ceil(max_h);
  for (size_t i = 0; i < nm; i++) {
    const uint64_t hgt = mats[i].height;
    ZKB_REQUIRE(hgt > 0, "matrix height 0 not supported");
    const int bits_reduced = log_max - log2_ceil(hgt);
    const uint64_t expected = ((max_h - 1) >> bits_reduced) + 1;
    ZKB_REQUIRE(hgt == expected, "matrix height %llu incompatible with tallest height %llu",
                (unsigned long long)hgt, (unsigned long long)max_h);
  }
  for (size_t i = 0; i + 1 < nm; i++) {
    uint64_t a = mats[ord[i]].height, b = mats[ord[i + 1]].height;
    ZKB_REQUIRE(a == b || next_pow2_u64(a) != next_pow2_u64(b),
                "matrix heights that round up to the same power of two must be equal");
  }

  // layer lengths
  t->layer_len.clear();
  t->layer_off.clear();
  uint64_t len = max_h == 1 ? 1 : max_h + (max_h & 1), total = 0;
  for (;;) {
    t->layer_off.push_back(total);
    t->layer_len.push_back(len);
    total += len;
    if (len == 1) break;
    len = len == 2 ? 1 : ((len / 2 + 1) & ~1ull);
  }
  t->spec = h;
  t->stream = s;
  t->device = ctx->device;
  t->mats = mats;
  ZKB_TRY(dev_alloc(&t->d_layers, total * OUT * sizeof(T), s));
  T *layers = (T *)t->d_layers;
  ZKB_CHECK_CUDA(cudaMemsetAsync(layers, 0, total * OUT * sizeof(T), s));

  auto make_list = [&](size_t first, size_t count, MatList *ml) -> int {
    ZKB_REQUIRE(count <= (size_t)MAX_GROUP_MATS, "more than %d matrices share one height",
                MAX_GROUP_MATS);
    ml->n = (int)count;
    ml->col_start[0] = 0;
    for (size_t i = 0; i < count; i++) {
      const TreeMatrix &m = mats[ord[first + i]];
      ml->ptr[i] = m.data;
      ml->width[i] = m.width;
      ml->col_start[i + 1] = ml->col_start[i] + m.width;
    }
    return ZKB_OK;
  };

  size_t ng = 0;
  while (ng < nm && mats[ord[ng]].height == max_h) ng++;
  MatList ml;
  ZKB_TRY(make_list(0, ng, &ml));
  const unsigned thr = 128;
  // One row (or pair) per thread and as many blocks as that takes: blocks retire every few
  // milliseconds, so kernels of other streams (other jobs of the engine, which gives small
  // jobs higher stream priority) get SMs in between instead of waiting for the whole grid.
  const unsigned cap = 1u << 30;
  (void)ctx;
  if (fill) {
    // the caller writes layer 0 (e.g. slab by slab as the matrix arrives)
    ZKB_REQUIRE(nm == 1 && comb == nullptr, "internal: leaves written by the caller take one matrix");
    ZKB_TRY((*fill)(layers));
  } else if constexpr (std::is_same<F, BabyBear>::value && W == 16) {
    if (comb) {
      ZKB_REQUIRE(nm == 1, "the fused alpha-reduction takes one matrix");
      ZKB_LAUNCH(leaf_name, s, hash_rows_combine_kernel<<<grid_for(max_h, thr, cap), thr, 0, s>>>((const uint32_t *)ml.ptr[0], ml.width[0], max_h, layers, p, comb->apow, comb->out));
    } else {
      ZKB_LAUNCH(leaf_name, s, hash_rows_kernel<F, W><<<grid_for(max_h, thr, cap), thr, 0, s>>>(ml, max_h, layers, p));
    }
  } else {
    ZKB_REQUIRE(comb == nullptr, "the fused alpha-reduction is BabyBear width 16 only");
    ZKB_LAUNCH(leaf_name, s, hash_rows_kernel<F, W><<<grid_for(max_h, thr, cap), thr, 0, s>>>(ml, max_h, layers, p));
  }
  ZKB_CHECK_LAUNCH();
  ScratchBuf inj_buf;  // digests of rows injected at one layer (sized for the largest)

  size_t next_m = ng;
  for (size_t li = 0; li + 1 < t->layer_len.size(); li++) {
    const uint64_t prev_len = t->layer_len[li];
    const uint64_t half = prev_len / 2;
    const uint64_t next_layer_len = next_pow2_u64(half);
    size_t ni = 0;
    while (next_m + ni < nm && next_pow2_u64(mats[ord[next_m + ni]].height) == next_layer_len) ni++;
    const T *prev = layers + t->layer_off[li] * OUT;
    T *next = layers + t->layer_off[li + 1] * OUT;
    const T *inj = nullptr;
    uint64_t inj_h = 0;
    if (ni) {
      MatList iml;
      ZKB_TRY(make_list(next_m, ni, &iml));
      inj_h = mats[ord[next_m]].height;
      if (!inj_buf.p) ZKB_TRY(inj_buf.alloc(inj_h * OUT * sizeof(T), s));
      ZKB_LAUNCH("merkle_inject_hash", s, hash_rows_kernel<F, W><<<grid_for(inj_h, thr, cap), thr, 0, s>>>(iml, inj_h, inj_buf.as<T>(), p));
      ZKB_CHECK_LAUNCH();
      inj = inj_buf.as<T>();
    }
    next_m += ni;
    ZKB_LAUNCH(comp_name, s, compress_kernel<F, W><<<grid_for(half, thr, cap), thr, 0, s>>>(prev, next, half, inj, inj_h, p));
    ZKB_CHECK_LAUNCH();
  }
  return ZKB_OK;
}

int mmcs_build_dev(const HasherSpec &h, const std::vector<TreeMatrix> &mats, DeviceTree *tree,
                   cudaStream_t s, bool fri_layer, const LeafCombine *comb, const LeafFill *fill) {
  ZKB_REQUIRE(!mats.empty(), "No matrices given");
  if (h.field == FIELD_BABYBEAR && h.width == 16) return build_tree_impl<BabyBear, 16>(h, mats, tree, s, fri_layer, comb, fill);
  if (h.field == FIELD_GOLDILOCKS && h.width == 16) return build_tree_impl<Goldilocks, 16>(h, mats, tree, s, fri_layer, comb, fill);
  if (h.field == FIELD_GOLDILOCKS && h.width == 12) return build_tree_impl<Goldilocks, 12>(h, mats, tree, s, fri_layer, comb, fill);
  set_error("unsupported hasher: field %d width %d", h.field, h.width);
  return ZKB_ERR_UNSUPPORTED;
}

int hash_rows_slab_dev(const HasherSpec &h, const uint32_t *mat, uint64_t stride, uint64_t c0, uint64_t ncols,
                       uint64_t height, uint32_t *carry, bool first, bool last, uint32_t *digests,
                       const LeafCombine *comb, cudaStream_t s) {
  ZKB_REQUIRE(h.field == FIELD_BABYBEAR && h.width == 16, "internal: slab leaf hashing is BabyBear width 16");
  ZKB_REQUIRE(c0 % 8 == 0 && (last || ncols % 8 == 0), "internal: slabs hold whole absorbed chunks");
  P2Params<BabyBear, 16> p;
  if (!build_p2_params<BabyBear, 16>(h, &p)) {
    set_error("invalid Poseidon2 parameters");
    return ZKB_ERR_INVALID;
  }
  const unsigned thr = 128;
  ZKB_LAUNCH("merkle_leaf_hash", s, hash_rows_slab_kernel<<<grid_for(height, thr, 1u << 30), thr, 0, s>>>(mat, stride, c0, ncols, height, carry, first ? 1 : 0, last ? 1 : 0, digests, p, comb ? comb->apow : nullptr, comb ? comb->out : nullptr));
  return ZKB_OK;
}

int mmcs_root_to_host(const DeviceTree *tree, void *root_out, cudaStream_t s) {
  const size_t es = field_elem_bytes(tree->spec.field);
  const uint64_t off = tree->layer_off.back() * tree->spec.out;
  ZKB_CHECK_CUDA(cudaMemcpyAsync(root_out, (const char *)tree->d_layers + off * es,
                                 tree->spec.out * es, cudaMemcpyDeviceToHost, s));
  ZKB_TRY(wait_stream(s));
  return ZKB_OK;
}

}  // namespace zkb
