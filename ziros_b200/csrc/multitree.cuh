// multitree.cuh — Merkle trees of many power-of-two-height matrices hashed together.
//
// One leaf-hash launch covers the rows of every matrix (job table + binary search of
// the job by row), one compression launch per level covers that level of every tree
// that still has it, and one launch gathers the roots.  Each tree is exactly the p3
// MerkleTree of its single matrix (vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:84-151:
// with a power-of-two height no layer is padded and nothing is injected), so a tree
// built here equals the one mmcs_build_dev builds for that matrix alone.  Used by the
// batched plan (many traces) and by the FRI commit phase (every round's layer tree).
#pragma once
#include <vector>

#include "common.cuh"
#include "poseidon2.cuh"

namespace zkb {
namespace mt {

struct LeafJob {
  const void *data;    // rows x width, row-major
  void *digests;       // rows x OUT (layer 0 of the job's tree)
  uint64_t row_start;  // prefix over the jobs
  uint64_t rows;
  uint64_t width;
};

struct CompJob {
  const void *prev;  // 2 * n_out digests
  void *next;        // n_out digests
  uint64_t start;    // prefix over the jobs of one level
  uint64_t n_out;
};

template <int W>
__host__ __device__ constexpr int digest_len() {
  return W == 16 ? 8 : 4;
}

// index of the last job whose start <= g (starts ascending, starts[0] = 0)
__device__ __forceinline__ int find_job(const uint64_t *starts, int n, uint64_t g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (starts[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// PaddingFreeSponge leaf digest of every row of every job (one permutation call site).
template <class F, int W>
__global__ void __launch_bounds__(256)
    mt_leaf_kernel(const LeafJob *__restrict__ jobs, int n_jobs, uint64_t total_rows,
                   const __grid_constant__ P2Params<F, W> p) {
  using T = typename F::T;
  using D = Dom<F>;
  constexpr int OUT = digest_len<W>();
  extern __shared__ uint64_t starts[];  // n_jobs entries
  for (int i = threadIdx.x; i < n_jobs; i += blockDim.x) starts[i] = jobs[i].row_start;
  __syncthreads();
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total_rows;
       g += (uint64_t)gridDim.x * blockDim.x) {
    const int j = find_job(starts, n_jobs, g);
    const uint64_t row = g - starts[j];
    const uint64_t width = jobs[j].width;
    const T *rp = (const T *)jobs[j].data + row * width;
    T s[W];
#pragma unroll
    for (int i = 0; i < W; i++) s[i] = 0;
    for (uint64_t c = 0; c < width; c += 8) {
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (c + i < width) s[i] = D::enter(rp[c + i]);
      p2_permute<F, W>(s, p);
    }
    T *out = (T *)jobs[j].digests + row * OUT;
#pragma unroll
    for (int i = 0; i < OUT; i++) out[i] = D::leave(s[i]);
  }
}

// next[i] = compress(prev[2i], prev[2i+1]) for every job of one tree level.
template <class F, int W>
__global__ void __launch_bounds__(128)
    mt_compress_kernel(const CompJob *__restrict__ jobs, int n_jobs, uint64_t total,
                       const __grid_constant__ P2Params<F, W> p) {
  using T = typename F::T;
  using D = Dom<F>;
  constexpr int OUT = digest_len<W>();
  extern __shared__ uint64_t starts[];  // n_jobs entries
  for (int i = threadIdx.x; i < n_jobs; i += blockDim.x) starts[i] = jobs[i].start;
  __syncthreads();
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (uint64_t)gridDim.x * blockDim.x) {
    const int j = find_job(starts, n_jobs, g);
    const uint64_t i = g - starts[j];
    const T *prev = (const T *)jobs[j].prev;
    T s[W];
#pragma unroll
    for (int k = 0; k < OUT; k++) {
      s[k] = D::enter(prev[(2 * i) * OUT + k]);
      s[OUT + k] = D::enter(prev[(2 * i + 1) * OUT + k]);
    }
#pragma unroll
    for (int k = 2 * OUT; k < W; k++) s[k] = 0;
    p2_permute<F, W>(s, p);
    T *next = (T *)jobs[j].next + i * OUT;
#pragma unroll
    for (int k = 0; k < OUT; k++) next[k] = D::leave(s[k]);
  }
}

// roots[dst[j]] = the last digest of job j's layers (offsets in digests from `base`;
// dst NULL: roots[j])
template <class T, int OUT>
__global__ void mt_roots_kernel(const uint64_t *__restrict__ root_off, const T *__restrict__ base, int n,
                                const uint32_t *__restrict__ dst, T *__restrict__ roots) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n * OUT) {
    const int j = t / OUT;
    roots[(uint64_t)(dst ? dst[j] : j) * OUT + (t % OUT)] = base[root_off[j] * OUT + (t % OUT)];
  }
}

// Host-side job tables of a set of trees.  layers[j] points at job j's digest layers
// (2 * rows - 1 digests, layer 0 first); root offsets are counted in digests from
// `base`, which must lie at or before every layers[j].
struct Tables {
  std::vector<LeafJob> leaf;
  std::vector<CompJob> comp;
  std::vector<size_t> lvl_off, lvl_cnt;
  std::vector<uint64_t> lvl_total;
  std::vector<uint64_t> root_off;
  std::vector<std::vector<uint64_t>> layer_len;
  uint64_t total_rows = 0;

  // device bytes of the tables (leaf jobs, compression jobs, root offsets)
  uint64_t device_bytes() const {
    return leaf.size() * sizeof(LeafJob) + comp.size() * sizeof(CompJob) + root_off.size() * 8;
  }
};

inline void build_tables(const std::vector<const void *> &data, const std::vector<uint64_t> &rows,
                         const std::vector<uint64_t> &width, const std::vector<void *> &layers, const void *base,
                         int out, size_t es, Tables *t) {
  const size_t n = data.size();
  *t = Tables{};
  t->leaf.resize(n);
  t->root_off.resize(n);
  t->layer_len.assign(n, {});
  size_t max_levels = 0;
  for (size_t i = 0; i < n; i++) {
    t->leaf[i] = LeafJob{data[i], layers[i], t->total_rows, rows[i], width[i]};
    t->total_rows += rows[i];
    uint64_t o = 0;
    for (uint64_t len = rows[i];; len /= 2) {
      t->layer_len[i].push_back(len);
      if (len == 1) break;
      o += len;
    }
    const uint64_t lay_off = (uint64_t)((const char *)layers[i] - (const char *)base) / (out * es);
    t->root_off[i] = lay_off + o;
    max_levels = std::max(max_levels, t->layer_len[i].size() - 1);
  }
  for (size_t l = 0; l < max_levels; l++) {
    t->lvl_off.push_back(t->comp.size());
    uint64_t start = 0;
    for (size_t i = 0; i < n; i++) {
      const auto &ll = t->layer_len[i];
      if (l + 1 >= ll.size()) continue;
      uint64_t lo = 0;
      for (size_t q = 0; q < l; q++) lo += ll[q];
      const char *lay = (const char *)layers[i];
      t->comp.push_back(CompJob{lay + lo * out * es, (void *)(lay + (lo + ll[l]) * out * es), start, ll[l] / 2});
      start += ll[l] / 2;
    }
    t->lvl_cnt.push_back(t->comp.size() - t->lvl_off.back());
    t->lvl_total.push_back(start);
  }
}

// Copies the tables into `dev` (device_bytes() bytes, 8-byte aligned) on stream s;
// returns the device addresses of the three parts.  The host tables must stay alive
// until the copies have been staged (pageable sources are staged before the call returns).
inline int upload_tables(const Tables &t, void *dev, cudaStream_t s, LeafJob **d_leaf, CompJob **d_comp,
                         uint64_t **d_root_off) {
  char *p = (char *)dev;
  *d_leaf = (LeafJob *)p;
  p += t.leaf.size() * sizeof(LeafJob);
  *d_comp = (CompJob *)p;
  p += t.comp.size() * sizeof(CompJob);
  *d_root_off = (uint64_t *)p;
  ZKB_CHECK_CUDA(cudaMemcpyAsync(*d_leaf, t.leaf.data(), t.leaf.size() * sizeof(LeafJob), cudaMemcpyHostToDevice, s));
  if (!t.comp.empty())
    ZKB_CHECK_CUDA(cudaMemcpyAsync(*d_comp, t.comp.data(), t.comp.size() * sizeof(CompJob), cudaMemcpyHostToDevice, s));
  ZKB_CHECK_CUDA(cudaMemcpyAsync(*d_root_off, t.root_off.data(), t.root_off.size() * 8, cudaMemcpyHostToDevice, s));
  return ZKB_OK;
}

// Enqueues the leaf hashing (unless the caller has written every job's leaf digests
// already: leaf_name NULL), every compression level and the root gather on s.
template <class F, int W>
int launch_trees(const Tables &t, const LeafJob *d_leaf, const CompJob *d_comp, const uint64_t *d_root_off,
                 const void *base, void *d_roots, const P2Params<F, W> &p, unsigned leaf_threads,
                 cudaStream_t s, const char *leaf_name, const char *comp_name, const char *root_name,
                 const uint32_t *d_root_dst = nullptr) {
  using T = typename F::T;
  constexpr int OUT = digest_len<W>();
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));
  const int n = (int)t.leaf.size();
  // one row (or compression) per thread: short-lived blocks, so concurrent streams
  // interleave at block granularity
  (void)ctx;
  if (leaf_name)
    ZKB_LAUNCH(leaf_name, s, mt_leaf_kernel<F, W><<<grid_for(t.total_rows, leaf_threads, 1u << 30), leaf_threads, n * sizeof(uint64_t), s>>>(d_leaf, n, t.total_rows, p));
  for (size_t l = 0; l < t.lvl_cnt.size(); l++) {
    ZKB_LAUNCH(comp_name, s, mt_compress_kernel<F, W><<<grid_for(t.lvl_total[l], 128, 1u << 30), 128, t.lvl_cnt[l] * sizeof(uint64_t), s>>>(d_comp + t.lvl_off[l], (int)t.lvl_cnt[l], t.lvl_total[l], p));
  }
  ZKB_LAUNCH(root_name, s, mt_roots_kernel<T, OUT><<<(n * OUT + 127) / 128, 128, 0, s>>>(d_root_off, (const T *)base, n, d_root_dst, (T *)d_roots));
  return ZKB_OK;
}

}  // namespace mt
}  // namespace zkb
