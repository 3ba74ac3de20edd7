// runtime.cu — a CUDA dispatch driver for the prover runtime's graph nodes.
//
// The reference runtime schedules a graph of ProverOp nodes over buffer slots and hands
// GPU-placed nodes to a GpuDispatchDriver (zkf-runtime/src/metal_driver.rs:55-80, op set
// zkf-runtime/src/graph.rs:51-110, Metal implementation
// zkf-runtime/src/metal_dispatch_macos.rs:150-400), which runs the node or returns a
// FallbackSignal so the node runs on the CPU.  This is that driver for the commitment
// path: device buffer slots, nodes Ntt / Lde / PoseidonBatch / MerkleLayer (a whole
// tree) / FriFold / FriQueryOpen with explicit dependencies on earlier nodes, executed
// in order on one stream with per-node device time.  A node the device path declines
// (the library's thresholds, kill switch or open circuit) stops the run and names the
// node, the reference's fallback signal.  The Lde node is one the Metal driver lacks.
#include <memory>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

namespace zkb {
namespace {

// Rows of a committed matrix and their sibling paths, one thread per query.  The indices
// live in a device buffer the host has not seen: a query whose index is past the tree
// opens nothing and records itself in *bad (the smallest such query number), which the
// host reads and reports as an error.
template <class T, int OUT>
__global__ void open_rows_kernel(const T *__restrict__ leaves, uint64_t rows, uint32_t width,
                                 const T *__restrict__ layers, const uint64_t *__restrict__ layer_off, int depth,
                                 const uint64_t *__restrict__ idx, int n, T *__restrict__ out,
                                 unsigned long long *bad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const uint64_t i = idx[q];
  if (i >= rows) {
    atomicMin(bad, (unsigned long long)q);
    return;
  }
  T *o = out + (uint64_t)q * (width + (uint64_t)depth * OUT);
  for (uint32_t c = 0; c < width; c++) o[c] = leaves[i * width + c];
  for (int l = 0; l < depth; l++) {
    const uint64_t j = (i >> l) ^ 1ull;
    for (int k = 0; k < OUT; k++) o[width + l * OUT + k] = layers[(layer_off[l] + j) * OUT + k];
  }
}

}  // namespace
}  // namespace zkb

using namespace zkb;

struct zkb_rt {
  int device = 0;
  cudaStream_t own = nullptr;
  std::vector<std::pair<void *, uint64_t>> bufs;
  std::vector<zkb_rt_node> nodes;
  std::vector<std::vector<int>> deps;
  std::vector<std::unique_ptr<zkb_tree>> trees;  // per node (Merkle nodes only)
  std::vector<float> node_ms;

  ~zkb_rt() {
    cudaSetDevice(device);
    if (own) cudaStreamSynchronize(own);
    trees.clear();
    for (auto &b : bufs) cudaFree(b.first);
    if (own) cudaStreamDestroy(own);
  }

  int slot(int id, uint64_t need, void **p) {
    ZKB_REQUIRE(id >= 0 && id < (int)bufs.size(), "unknown buffer slot %d", id);
    ZKB_REQUIRE(bufs[id].second >= need, "buffer slot %d holds %llu bytes, the node needs %llu", id,
                (unsigned long long)bufs[id].second, (unsigned long long)need);
    *p = bufs[id].first;
    return ZKB_OK;
  }

  // the driver's placement test (the reference's should_try_on_either with thresholds,
  // zkf-runtime/src/metal_dispatch_macos.rs:170-186)
  static int placement(const zkb_rt_node &n) {
    const zkb_thresholds t = thresholds();
    const uint64_t rows = 1ull << n.log_n;
    switch (n.kind) {
      case ZKB_OP_NTT:
      case ZKB_OP_LDE: return below(rows, t.ntt, "ntt");
      case ZKB_OP_POSEIDON_BATCH: return below(n.count, t.poseidon2, "poseidon2");
      case ZKB_OP_MERKLE: return below(rows, t.merkle, "merkle");
      case ZKB_OP_FRI_FOLD: return below(rows / 2, t.fri, "fri");
      default: return ZKB_OK;
    }
  }

  template <class F>
  int run_field(int id, const zkb_rt_node &n, cudaStream_t s) {
    using T = typename F::T;
    const size_t es = sizeof(T);
    const uint64_t rows = 1ull << n.log_n;
    void *in = nullptr, *out = nullptr;
    ZKB_REQUIRE(n.log_n < 40, "log_n too large");
    switch (n.kind) {
      case ZKB_OP_NTT: {
        ZKB_TRY(slot(n.in_slot, rows * n.width * es, &in));
        return ntt_dft_dev<F>((T *)in, (int)n.log_n, n.width, n.inverse != 0, s);
      }
      case ZKB_OP_LDE: {
        ZKB_TRY(slot(n.in_slot, rows * n.width * es, &in));
        ZKB_TRY(slot(n.out_slot, (rows << n.log_blowup) * n.width * es, &out));
        return ntt_lde_dev<F>((const T *)in, (int)n.log_n, n.width, (int)n.log_blowup, F::GENERATOR, true,
                              (T *)out, s);
      }
      case ZKB_OP_POSEIDON_BATCH: {
        ZKB_TRY(slot(n.in_slot, n.count * 16 * es, &in));
        HasherSpec spec;
        ZKB_REQUIRE(make_hasher_spec(n.field, 16, n.seed, &spec), "unsupported hasher");
        P2Params<F, 16> p;
        ZKB_REQUIRE((build_p2_params<F, 16>(spec, &p)), "invalid Poseidon2 parameters");
        return p2_permute_batch<F, 16>((T *)in, n.count, p, s);
      }
      case ZKB_OP_MERKLE: {
        ZKB_TRY(slot(n.in_slot, rows * n.width * es, &in));
        HasherSpec spec;
        ZKB_REQUIRE(make_hasher_spec(n.field, n.hasher_width ? (int)n.hasher_width : 16, n.seed, &spec),
                    "unsupported hasher");
        auto t = std::make_unique<zkb_tree>();
        std::vector<TreeMatrix> m{{in, rows, n.width}};
        ZKB_TRY(mmcs_build_dev(spec, m, &t->t, s));
        if (n.out_slot >= 0) {
          ZKB_TRY(slot(n.out_slot, spec.out * es, &out));
          const DeviceTree &dt = t->t;
          ZKB_CHECK_CUDA(cudaMemcpyAsync(out, (const char *)dt.d_layers + dt.layer_off.back() * spec.out * es,
                                         spec.out * es, cudaMemcpyDeviceToDevice, s));
        }
        trees[id] = std::move(t);
        return ZKB_OK;
      }
      case ZKB_OP_FRI_FOLD: {
        // fold of 2^log_n evaluations: F_p^4 (ext4, BabyBear) or base field, p3 fold_matrix
        if (n.ext4) {
          ZKB_REQUIRE(n.field == ZKB_FIELD_BABYBEAR, "the F_p^4 fold is over BabyBear");
          ZKB_TRY(slot(n.in_slot, rows * 16, &in));
          ZKB_TRY(slot(n.out_slot, rows / 2 * 16, &out));
          return fri_fold_ext4_dev((const uint32_t *)in, rows / 2, n.beta, (uint32_t *)out, s);
        }
        ZKB_TRY(slot(n.in_slot, rows * es, &in));
        ZKB_TRY(slot(n.out_slot, rows / 2 * es, &out));
        const T beta = sizeof(T) == 4 ? (T)n.beta[0] : (T)(((uint64_t)n.beta[1] << 32) | n.beta[0]);
        ZKB_REQUIRE(beta < F::P, "beta is not canonical");
        return fri_fold_base_dev<F>((const T *)in, rows / 2, beta, nullptr, (T *)out, s);
      }
      case ZKB_OP_FRI_QUERY_OPEN: {
        // opens n.count rows of the tree built by Merkle node n.tree_node at the indices in
        // in_slot (u64): out_slot gets, per query, the row then the sibling digests
        ZKB_REQUIRE(n.tree_node >= 0 && n.tree_node < id && trees[n.tree_node], "query node %d: node %d is not "
                    "an earlier Merkle node", id, n.tree_node);
        const DeviceTree &dt = trees[n.tree_node]->t;
        const uint64_t trows = dt.mats[0].height, tw = dt.mats[0].width;
        const int depth = (int)dt.layer_len.size() - 1;
        const int out_d = dt.spec.out;
        ZKB_TRY(slot(n.in_slot, n.count * 8, &in));
        ZKB_TRY(slot(n.out_slot, n.count * (tw + (uint64_t)depth * out_d) * es, &out));
        if (n.count == 0) return ZKB_OK;
        ZKB_REQUIRE(n.count <= 0x7fffffffull, "query node %d: %llu queries", id, (unsigned long long)n.count);
        // scratch: the layer offsets, then the bad-query word (all ones: none)
        ScratchBuf d_off;
        ZKB_TRY(d_off.alloc((depth + 2) * 8, s));
        std::vector<uint64_t> hbuf(dt.layer_off.begin(), dt.layer_off.begin() + depth + 1);
        hbuf.push_back(~0ull);
        ZKB_CHECK_CUDA(cudaMemcpyAsync(d_off.p, hbuf.data(), (depth + 2) * 8, cudaMemcpyHostToDevice, s));
        unsigned long long *d_bad = reinterpret_cast<unsigned long long *>(d_off.as<uint64_t>() + depth + 1);
        const unsigned grid = (unsigned)((n.count + 127) / 128);
        if (out_d == 8)
          ZKB_LAUNCH("rt_query_open", s, open_rows_kernel<T, 8><<<grid, 128, 0, s>>>((const T *)dt.mats[0].data, trows, (uint32_t)tw, (const T *)dt.d_layers, d_off.as<uint64_t>(), depth, (const uint64_t *)in, (int)n.count, (T *)out, d_bad));
        else
          ZKB_LAUNCH("rt_query_open", s, open_rows_kernel<T, 4><<<grid, 128, 0, s>>>((const T *)dt.mats[0].data, trows, (uint32_t)tw, (const T *)dt.d_layers, d_off.as<uint64_t>(), depth, (const uint64_t *)in, (int)n.count, (T *)out, d_bad));
        unsigned long long bad = 0;
        ZKB_CHECK_CUDA(cudaMemcpyAsync(&bad, d_bad, 8, cudaMemcpyDeviceToHost, s));
        // the layer offsets and the bad-query word are read before the scratch is released
        ZKB_TRY(wait_stream(s));
        if (bad != ~0ull) {
          uint64_t bad_idx = 0;
          ZKB_CHECK_CUDA(cudaMemcpy(&bad_idx, (const uint64_t *)in + bad, 8, cudaMemcpyDeviceToHost));
          set_error("query node %d: query %llu opens row %llu of a %llu-row tree", id, bad,
                    (unsigned long long)bad_idx, (unsigned long long)trows);
          return ZKB_ERR_INVALID;
        }
        return ZKB_OK;
      }
      default:
        set_error("unknown node kind %d", n.kind);
        return ZKB_ERR_INVALID;
    }
  }
};

extern "C" {

int zkb_rt_create(zkb_rt **out) {
  clear_error();
  ZKB_REQUIRE(out != nullptr, "null output");
  ZKB_TRY(library_gate());
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) {
    set_error("no CUDA device available");
    return ZKB_DECLINED;
  }
  auto rt = std::make_unique<zkb_rt>();
  ZKB_CHECK_CUDA(cudaGetDevice(&rt->device));
  ZKB_CHECK_CUDA(cudaStreamCreateWithFlags(&rt->own, cudaStreamNonBlocking));
  *out = rt.release();
  return ZKB_OK;
}

int zkb_rt_buffer(zkb_rt *rt, uint64_t bytes, int *slot_out) {
  clear_error();
  ZKB_REQUIRE(rt && slot_out && bytes > 0, "invalid arguments");
  ZKB_CHECK_CUDA(cudaSetDevice(rt->device));
  void *p = nullptr;
  note_device_alloc();
  ZKB_CHECK_CUDA(cudaMalloc(&p, bytes));
  rt->bufs.emplace_back(p, bytes);
  *slot_out = (int)rt->bufs.size() - 1;
  return ZKB_OK;
}

int zkb_rt_write(zkb_rt *rt, int slot, const void *host, uint64_t bytes) {
  clear_error();
  ZKB_REQUIRE(rt && host, "null arguments");
  void *p;
  ZKB_TRY(rt->slot(slot, bytes, &p));
  ZKB_CHECK_CUDA(cudaMemcpyAsync(p, host, bytes, cudaMemcpyHostToDevice, rt->own));
  return wait_stream(rt->own);
}

int zkb_rt_read(zkb_rt *rt, int slot, void *host, uint64_t bytes) {
  clear_error();
  ZKB_REQUIRE(rt && host, "null arguments");
  void *p;
  ZKB_TRY(rt->slot(slot, bytes, &p));
  ZKB_CHECK_CUDA(cudaMemcpyAsync(host, p, bytes, cudaMemcpyDeviceToHost, rt->own));
  return wait_stream(rt->own);
}

int zkb_rt_add(zkb_rt *rt, const zkb_rt_node *node, const int *deps, size_t n_deps, int *node_id) {
  clear_error();
  ZKB_REQUIRE(rt && node && node_id && (deps || n_deps == 0), "null arguments");
  ZKB_REQUIRE(node->field == ZKB_FIELD_BABYBEAR || node->field == ZKB_FIELD_GOLDILOCKS, "unknown field");
  const int id = (int)rt->nodes.size();
  for (size_t i = 0; i < n_deps; i++)
    ZKB_REQUIRE(deps[i] >= 0 && deps[i] < id, "node %d depends on node %d, which is not an earlier node", id,
                deps[i]);
  rt->nodes.push_back(*node);
  rt->deps.emplace_back(deps, deps + n_deps);
  rt->trees.emplace_back();
  rt->node_ms.push_back(0.f);
  *node_id = id;
  return ZKB_OK;
}

int zkb_rt_execute(zkb_rt *rt, void *stream, int *fallback_node) {
  clear_error();
  ZKB_REQUIRE(rt != nullptr, "null runtime");
  if (fallback_node) *fallback_node = -1;
  ZKB_CHECK_CUDA(cudaSetDevice(rt->device));
  cudaStream_t s = stream ? resolve_stream(stream) : rt->own;
  // nodes only depend on earlier nodes, so insertion order is a topological order and one
  // stream keeps every dependency; a node whose inputs are not ready cannot exist
  std::vector<cudaEvent_t> ev(2 * rt->nodes.size(), nullptr);
  for (auto &e : ev) ZKB_CHECK_CUDA(cudaEventCreate(&e));
  int rc = ZKB_OK;
  size_t i = 0;
  for (; i < rt->nodes.size() && rc == ZKB_OK; i++) {
    rc = library_gate();
    if (rc != ZKB_OK) break;
    const zkb_rt_node &n = rt->nodes[i];
    rc = zkb_rt::placement(n);
    if (rc != ZKB_OK) break;
    cudaEventRecord(ev[2 * i], s);
    rc = n.field == ZKB_FIELD_BABYBEAR ? rt->run_field<BabyBear>((int)i, n, s)
                                       : rt->run_field<Goldilocks>((int)i, n, s);
    cudaEventRecord(ev[2 * i + 1], s);
  }
  if (rc == ZKB_DECLINED && fallback_node) *fallback_node = (int)i;
  if (rc != ZKB_OK && fallback_node && *fallback_node < 0) *fallback_node = (int)(i ? i - 1 : 0);
  const int wrc = wait_stream(s);
  if (rc == ZKB_OK && wrc == ZKB_OK)
    for (size_t k = 0; k < rt->nodes.size(); k++) cudaEventElapsedTime(&rt->node_ms[k], ev[2 * k], ev[2 * k + 1]);
  for (auto e : ev) cudaEventDestroy(e);
  return rc != ZKB_OK ? rc : wrc;
}

int zkb_rt_node_ms(const zkb_rt *rt, int node_id, float *ms) {
  clear_error();
  ZKB_REQUIRE(rt && ms && node_id >= 0 && node_id < (int)rt->nodes.size(), "invalid node");
  *ms = rt->node_ms[node_id];
  return ZKB_OK;
}

int zkb_rt_tree(const zkb_rt *rt, int node_id, const zkb_tree **tree) {
  clear_error();
  ZKB_REQUIRE(rt && tree && node_id >= 0 && node_id < (int)rt->trees.size() && rt->trees[node_id],
              "node %d has no tree (not a Merkle node, or not executed)", node_id);
  *tree = rt->trees[node_id].get();
  return ZKB_OK;
}

void zkb_rt_free(zkb_rt *rt) { delete rt; }

}  // extern "C"
