// batch.cu — batched commitment of many traces of uneven height and width.
//
// A plan (zkb_batch_create) owns one device arena with every trace's input, LDE and
// digest layers, builds the twiddle and coset tables, and chooses kernel shapes
// (autotuned and cached, or defaults).  A run is one CUDA graph:
//
//   fork -> per branch, the coset LDEs of its traces (ntt passes + fused middle kernel,
//           coefficient scratch owned by the branch)
//   join -> ONE leaf-hash launch over the rows of all traces (job table, binary search
//           of the trace by row)
//        -> one compression launch per tree level, across every tree that still has
//           that level
//        -> one launch gathering the roots
//
// With use_graph = 2 (BabyBear, widths that are multiples of 8) a run is instead ONE
// persistent kernel fed by a device work queue (persist.cu), captured in the graph: every
// trace's NTT passes, leaf hashing and compression levels are items that the kernel's
// blocks claim in order, each waiting (bounded) for the step it depends on; the
// autotuner then also chooses the Merkle-level fusion (levels computed in shared memory by
// the tile that made the level below).
//
// Every trace gets exactly the p3 MerkleTree of its own LDE (power-of-two heights: no
// padding, no injection), so each root equals the plain per-trace commitment
// (TwoAdicFriPcs::commit over one matrix, vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:84-151).
// The reference commits each trace with its own dispatch sequence; the plan is this
// library's batched form of that call.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "multitree.cuh"
#include "persist.cuh"
#include "poseidon2.cuh"

namespace zkb {
namespace {

constexpr int MAX_BATCH = 1024;
using mt::CompJob;
using mt::LeafJob;

// Job tables of a set of trees: host copy and device pointers (root_dst: the batch index
// of each root, NULL when the set is the whole batch in order).
struct JobTables {
  mt::Tables t;
  const LeafJob *leaf = nullptr;
  const CompJob *comp = nullptr;
  const uint64_t *root_off = nullptr;
  const uint32_t *root_dst = nullptr;
};

// A group of a run from host memory: traces consecutive in the copy order (smallest
// first), committed together once their copies have landed — their LDEs over the
// branches, then one multi-tree launch set — as one graph (or the same launches).
struct HostGroup {
  std::vector<int> traces;
  std::vector<char> member;  // per batch index
  int lane = 0;              // 0: the caller's stream and the plan's scratch, 1: the second lane
  JobTables jobs;
  cudaEvent_t copied = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }

uint64_t fnv1a(const void *data, size_t n, uint64_t h = 1469598103934665603ull) {
  const unsigned char *p = (const unsigned char *)data;
  for (size_t i = 0; i < n; i++) h = (h ^ p[i]) * 1099511628211ull;
  return h;
}

// ---- tuning cache: one JSON object per line, {"key": "...", "name": int, ...}
struct TuneCache {
  std::string path;
  std::vector<std::pair<std::string, std::string>> lines;  // key, full line

  void load() {
    if (path.empty()) return;
    std::ifstream f(path);
    std::string ln;
    while (std::getline(f, ln)) {
      const size_t k = ln.find("\"key\": \"");
      if (k == std::string::npos) continue;
      const size_t a = k + 8, b = ln.find('"', a);
      if (b == std::string::npos) continue;
      lines.emplace_back(ln.substr(a, b - a), ln);
    }
  }
  const std::string *find(const std::string &key) const {
    for (auto &kv : lines)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
  static bool field(const std::string &line, const char *name, long *out) {
    const std::string pat = std::string("\"") + name + "\": ";
    const size_t k = line.find(pat);
    if (k == std::string::npos) return false;
    *out = strtol(line.c_str() + k + pat.size(), nullptr, 10);
    return true;
  }
  void put(const std::string &key, const std::string &line) {
    for (auto &kv : lines)
      if (kv.first == key) {
        kv.second = line;
        return;
      }
    lines.emplace_back(key, line);
  }
  void save() const {
    if (path.empty()) return;
    const std::string tmp = path + ".tmp";
    {
      std::ofstream f(tmp, std::ios::trunc);
      if (!f) return;
      for (auto &kv : lines) f << kv.second << "\n";
    }
    std::rename(tmp.c_str(), path.c_str());
  }
};

}  // namespace
}  // namespace zkb

using namespace zkb;

struct zkb_batch {
  int device = 0;
  HasherSpec spec;
  uint32_t log_b = 1;
  size_t es = 4;
  int out = 8;
  std::vector<zkb_batch_shape> shapes;
  // arena
  void *arena = nullptr;
  uint64_t arena_bytes = 0;
  std::vector<void *> d_in, d_lde, d_layers;
  std::vector<void *> d_coef;                    // per branch: scratch for its largest trace
  uint64_t coef_bytes = 0;
  void *d_roots = nullptr;
  JobTables joint;  // every trace's tree, roots in batch order
  // kernel shapes
  std::vector<LdeTune> tune;  // per trace
  unsigned leaf_threads = 128;
  uint32_t branches = 1;
  std::vector<std::vector<int>> branch_traces;
  bool use_graph = true;
  bool persistent = false;             // one persistent kernel per run (use_graph = 2)
  std::unique_ptr<PersistPlan> persist;
  void *d_coef_all = nullptr;          // persistent form: coefficient scratch slots
  std::vector<uint32_t *> coef_of;     // per trace: its slot
  std::vector<int> slot_prev, round_of, queue_order;
  uint32_t coef_slots = 0;
  MerkleFusion fusion{3, 4};
  bool tuned_from_cache = false;
  double tune_ms = 0;
  // execution
  cudaStream_t s_main = nullptr;
  std::vector<cudaStream_t> s_br;
  std::vector<cudaEvent_t> ev_br;
  cudaEvent_t ev_fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t kernels_per_run = 0;
  // runs from host memory (run_host): copy stream and the groups of the copy order
  cudaStream_t s_copy = nullptr;
  cudaEvent_t ev_host = nullptr, ev_copied = nullptr;
  std::vector<HostGroup> host_groups;
  // a second lane for the host groups: its own stream and a second coefficient-scratch set,
  // so that a group's LDEs overlap the tail of the group before it (graph plans only)
  uint32_t host_lanes = 1;
  bool host_ready = false;  // lanes set up and group graphs captured (at the first run_host)
  cudaStream_t s_lane = nullptr;
  cudaEvent_t ev_lane = nullptr;
  void *d_coef2_base = nullptr;
  std::vector<void *> d_coef2;
  P2Params<BabyBear, 16> p_bb16;
  P2Params<Goldilocks, 16> p_gl16;
  P2Params<Goldilocks, 12> p_gl12;
  std::vector<std::unique_ptr<zkb_tree>> trees;

  ~zkb_batch() {
    cudaSetDevice(device);
    if (s_main) cudaStreamSynchronize(s_main);
    trees.clear();
    if (!d_coef.empty()) cudaFree(d_coef[0]);
    persist.reset();
    if (d_coef_all) cudaFree(d_coef_all);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto e : ev_br) cudaEventDestroy(e);
    for (auto &g : host_groups) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      if (g.graph) cudaGraphDestroy(g.graph);
      if (g.copied) cudaEventDestroy(g.copied);
    }
    if (ev_host) cudaEventDestroy(ev_host);
    if (ev_copied) cudaEventDestroy(ev_copied);
    if (ev_lane) cudaEventDestroy(ev_lane);
    if (s_lane) cudaStreamDestroy(s_lane);
    if (d_coef2_base) cudaFree(d_coef2_base);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (s_copy) cudaStreamDestroy(s_copy);
    for (auto s : s_br) cudaStreamDestroy(s);
    if (s_main) cudaStreamDestroy(s_main);
    if (arena) cudaFree(arena);
  }

  uint64_t rows_of(size_t i) const { return 1ull << (shapes[i].log_h + log_b); }

  // ---- launches of one run, enqueued on `origin` (captured or direct)
  int lde_one(size_t i, cudaStream_t s, const LdeTune *t, int lane = 0) {
    const int lh = (int)shapes[i].log_h;
    const uint32_t w = shapes[i].width;
    const int br = branch_of(i);
    void *scratch = lane ? d_coef2[br] : d_coef[br];
    if (spec.field == FIELD_BABYBEAR)
      return ntt_lde_dev<BabyBear>((const uint32_t *)d_in[i], lh, w, (int)log_b, BabyBear::GENERATOR, true,
                                   (uint32_t *)d_lde[i], s, t, (uint32_t *)scratch);
    return ntt_lde_dev<Goldilocks>((const uint64_t *)d_in[i], lh, w, (int)log_b, Goldilocks::GENERATOR, true,
                                   (uint64_t *)d_lde[i], s, t, (uint64_t *)scratch);
  }
  int branch_of(size_t i) const {
    for (size_t b = 0; b < branch_traces.size(); b++)
      for (int t : branch_traces[b])
        if ((size_t)t == i) return (int)b;
    return 0;
  }

  // The trees of a set of traces: one leaf-hash launch over all their rows, one
  // compression launch per level, one root gather.
  template <class F, int W>
  int hash_set(const JobTables &j, const P2Params<F, W> &p, unsigned threads, cudaStream_t s) {
    return mt::launch_trees<F, W>(j.t, j.leaf, j.comp, j.root_off, d_layers[0], d_roots, p, threads, s,
                                  "batch_leaf_hash", "batch_compress", "batch_roots", j.root_dst);
  }

  int hash_tables(const JobTables &j, unsigned threads, cudaStream_t s) {
    if (spec.field == FIELD_BABYBEAR) return hash_set<BabyBear, 16>(j, p_bb16, threads, s);
    if (spec.width == 16) return hash_set<Goldilocks, 16>(j, p_gl16, threads, s);
    return hash_set<Goldilocks, 12>(j, p_gl12, threads, s);
  }

  int hash_dispatch(unsigned threads, cudaStream_t s) { return hash_tables(joint, threads, s); }

  // The LDEs of the `member` traces (every trace when NULL), forked over their branches
  // (each branch in its own order, with its own coefficient scratch of the lane's set) and
  // joined on origin.
  int enqueue_ldes(const std::vector<char> *member, cudaStream_t origin, int lane = 0) {
    const uint32_t nb = (uint32_t)branch_traces.size();
    ZKB_CHECK_CUDA(cudaEventRecord(ev_fork, origin));
    for (uint32_t b = 0; b < nb; b++) {
      bool any = !member;
      for (int i : branch_traces[b]) any = any || (*member)[i];
      if (!any) continue;
      ZKB_CHECK_CUDA(cudaStreamWaitEvent(s_br[b], ev_fork, 0));
      for (int i : branch_traces[b])
        if (!member || (*member)[i]) ZKB_TRY(lde_one((size_t)i, s_br[b], &tune[i], lane));
      ZKB_CHECK_CUDA(cudaEventRecord(ev_br[b], s_br[b]));
      ZKB_CHECK_CUDA(cudaStreamWaitEvent(origin, ev_br[b], 0));
    }
    return ZKB_OK;
  }

  int enqueue_group(const HostGroup &g, cudaStream_t origin) {
    ZKB_TRY(enqueue_ldes(&g.member, origin, g.lane));
    return hash_tables(g.jobs, leaf_threads, origin);
  }

  // A second coefficient-scratch set (each branch's largest trace again) when it takes at
  // most an eighth of free device memory: the host groups then alternate between two lanes.
  int setup_host_lanes() {
    host_lanes = 1;
    if (host_groups.size() < 2) return ZKB_OK;
    std::vector<uint64_t> need(branch_traces.size(), 0);
    uint64_t total = 0;
    for (size_t b = 0; b < branch_traces.size(); b++) {
      for (int i : branch_traces[b]) need[b] = std::max<uint64_t>(need[b], (1ull << shapes[i].log_h) * shapes[i].width * es);
      need[b] = align256(std::max<uint64_t>(need[b], 256));
      total += need[b];
    }
    size_t free_b = 0, total_b = 0;
    ZKB_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (total > free_b / 8) {
      for (auto &g : host_groups) g.lane = 0;
      return ZKB_OK;
    }
    note_device_alloc();
    if (cudaMalloc(&d_coef2_base, total) != cudaSuccess) {  // one lane, then
      cudaGetLastError();
      d_coef2_base = nullptr;
      for (auto &g : host_groups) g.lane = 0;
      return ZKB_OK;
    }
    d_coef2.assign(branch_traces.size(), nullptr);
    uint64_t o = 0;
    for (size_t b = 0; b < branch_traces.size(); b++) {
      d_coef2[b] = (char *)d_coef2_base + o;
      o += need[b];
    }
    ZKB_CHECK_CUDA(cudaStreamCreateWithFlags(&s_lane, cudaStreamNonBlocking));
    ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&ev_lane, cudaEventDisableTiming));
    for (size_t k = 0; k < host_groups.size(); k++) host_groups[k].lane = (int)(k % 2);
    host_lanes = 2;
    return ZKB_OK;
  }

  // One graph per host group (the group's launches captured on s_main).
  int capture_groups() {
    for (auto &g : host_groups) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      if (g.graph) cudaGraphDestroy(g.graph);
      g.exec = nullptr;
      g.graph = nullptr;
      ZKB_CHECK_CUDA(cudaStreamBeginCapture(s_main, cudaStreamCaptureModeRelaxed));
      const int rc = enqueue_group(g, s_main);
      cudaGraph_t gr = nullptr;
      const cudaError_t e = cudaStreamEndCapture(s_main, &gr);
      ZKB_TRY(rc);
      if (e != cudaSuccess) {
        set_error("graph capture failed: %s", cudaGetErrorString(e));
        return ZKB_ERR_CUDA;
      }
      g.graph = gr;
      ZKB_CHECK_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
    }
    return ZKB_OK;
  }

  int copy_host(size_t i, const void *src, cudaStream_t s) {
    const uint64_t bytes = (1ull << shapes[i].log_h) * shapes[i].width * es;
    ZKB_CHECK_CUDA(cudaMemcpyAsync(d_in[i], src, bytes, cudaMemcpyHostToDevice, s));
    return ZKB_OK;
  }

  // A run whose traces come from host memory, the copies overlapped with the commitment:
  // the copy stream takes the traces in groups (about 1/64 of the batch's cells each, a
  // larger trace by itself), and each group's LDEs and trees run as soon as its last copy
  // has landed, while the next groups copy — the groups alternating between origin and a
  // second lane with its own scratch (when memory allows), so that a group's LDEs overlap
  // the small top levels of the trees of the group before it.  This is a two-stage flow (copy, then
  // compute) whose two stages run at similar rates per cell (the compute a little slower
  // or faster, depending on the host link): the work done outside the overlap is the
  // first group's copy and the last group's compute, so the copy order puts small traces
  // at both ends and the largest in the middle, growing gradually on the way up (a copy
  // then rarely outlasts the compute of the group before it) and shrinking on the way
  // down.  Copies and launches are enqueued group by group, so a pageable source (staged
  // by the copy call) still overlaps the staging of later groups with the work on earlier
  // ones.  A persistent plan reads every trace from its one kernel: its copies all go
  // first.
  int run_host(const void *const *src, cudaStream_t origin) {
    const size_t n = shapes.size();
    for (size_t i = 0; i < n; i++) ZKB_REQUIRE(src[i] != nullptr, "trace %zu: null host source", i);
    if (!persistent && !host_ready) {
      // set up at the first host run, so that plans never run from host memory keep the
      // memory and the creation time
      if (use_graph) {
        ZKB_TRY(setup_host_lanes());
        ZKB_TRY(capture_groups());
      }
      host_ready = true;
    }
    ZKB_CHECK_CUDA(cudaEventRecord(ev_host, origin));
    ZKB_CHECK_CUDA(cudaStreamWaitEvent(s_copy, ev_host, 0));
    if (host_lanes == 2) ZKB_CHECK_CUDA(cudaStreamWaitEvent(s_lane, ev_host, 0));
    int rc = ZKB_OK;
    if (persistent) {
      for (size_t i = 0; i < n && rc == ZKB_OK; i++) rc = copy_host(i, src[i], s_copy);
    } else {
      for (size_t k = 0; k < host_groups.size() && rc == ZKB_OK; k++) {
        HostGroup &g = host_groups[k];
        for (size_t q = 0; q < g.traces.size() && rc == ZKB_OK; q++) rc = copy_host(g.traces[q], src[g.traces[q]], s_copy);
        if (rc != ZKB_OK) break;
        cudaStream_t ls = g.lane ? s_lane : origin;
        if (cudaEventRecord(g.copied, s_copy) != cudaSuccess || cudaStreamWaitEvent(ls, g.copied, 0) != cudaSuccess) {
          set_error("copy ordering failed: %s", cudaGetErrorString(cudaGetLastError()));
          rc = ZKB_ERR_CUDA;
          break;
        }
        if (g.exec) {
          if (cudaGraphLaunch(g.exec, ls) != cudaSuccess) {
            set_error("group graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            rc = ZKB_ERR_CUDA;
          }
        } else {
          rc = enqueue_group(g, ls);
        }
      }
    }
    // origin joins the second lane and the copy stream, also after an error (the sources are
    // read until then)
    if (host_lanes == 2) {
      ZKB_CHECK_CUDA(cudaEventRecord(ev_lane, s_lane));
      ZKB_CHECK_CUDA(cudaStreamWaitEvent(origin, ev_lane, 0));
    }
    ZKB_CHECK_CUDA(cudaEventRecord(ev_copied, s_copy));
    ZKB_CHECK_CUDA(cudaStreamWaitEvent(origin, ev_copied, 0));
    ZKB_TRY(rc);
    return persistent ? persist->enqueue(origin) : ZKB_OK;
  }

  // The persistent form's plan over the current kernel shapes and Merkle fusion.
  int build_persist() {
    // the plan's traces in queue order (largest first); slot_prev refers to that order
    std::vector<PersistTrace> tr(shapes.size());
    for (size_t k = 0; k < shapes.size(); k++) {
      const size_t i = (size_t)queue_order[k];
      tr[k].slot_prev = slot_prev[k];
      tr[k].round = round_of[k];
      tr[k].in = (const uint32_t *)d_in[i];
      tr[k].coef = coef_of[i];
      tr[k].lde = (uint32_t *)d_lde[i];
      tr[k].layers = (uint32_t *)d_layers[i];
      tr[k].root = (uint32_t *)d_roots + i * 8;
      tr[k].log_h = (int)shapes[i].log_h;
      tr[k].width = shapes[i].width;
      tr[k].kmax = std::min(tune[i].kmax ? tune[i].kmax : 9, 9);
    }
    auto plan = std::make_unique<PersistPlan>();
    ZKB_TRY(plan->build(tr, (int)log_b, p_bb16, fusion, s_main));
    persist = std::move(plan);
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    return ZKB_OK;
  }

  int enqueue(cudaStream_t origin) {
    if (persistent) return persist->enqueue(origin);
    ZKB_TRY(enqueue_ldes(nullptr, origin));
    return hash_dispatch(leaf_threads, origin);
  }

  // Longest-processing-time assignment of the traces to `nb` branches; each branch gets
  // coefficient scratch for its largest trace.  Fails (without changing the current
  // assignment) when that scratch does not fit in free device memory.
  int assign_branches(uint32_t nb) {
    std::vector<std::vector<int>> bt(nb);
    std::vector<int> ord(shapes.size());
    std::iota(ord.begin(), ord.end(), 0);
    auto cost = [&](int i) { return (double)rows_of(i) * shapes[i].width * (shapes[i].log_h + log_b + 1); };
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<double> load(nb, 0.0);
    for (int i : ord) {
      const size_t b = std::min_element(load.begin(), load.end()) - load.begin();
      bt[b].push_back(i);
      load[b] += cost(i);
    }
    std::vector<uint64_t> need(nb, 0);
    uint64_t total = 0;
    for (uint32_t b = 0; b < nb; b++) {
      for (int i : bt[b]) need[b] = std::max<uint64_t>(need[b], (1ull << shapes[i].log_h) * shapes[i].width * es);
      need[b] = align256(std::max<uint64_t>(need[b], 256));
      total += need[b];
    }
    size_t free_b = 0, total_b = 0;
    ZKB_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const uint64_t avail = free_b + coef_bytes;  // the current scratch is released first
    ZKB_REQUIRE(total + (1ull << 30) <= avail, "%u branches need %llu bytes of scratch, %llu available", nb,
                (unsigned long long)total, (unsigned long long)avail);
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    ZKB_TRY(wait_stream(s_main));
    if (!d_coef.empty()) cudaFree(d_coef[0]);
    d_coef.clear();
    coef_bytes = 0;
    void *scratch = nullptr;
    note_device_alloc();
    ZKB_CHECK_CUDA(cudaMalloc(&scratch, total));
    d_coef.push_back(scratch);
    for (uint32_t b = 1; b < nb; b++) d_coef.push_back((char *)d_coef[b - 1] + need[b - 1]);
    coef_bytes = total;
    branch_traces = std::move(bt);
    branches = nb;
    return ZKB_OK;
  }

  int capture() {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    if (graph) {
      cudaGraphDestroy(graph);
      graph = nullptr;
    }
    ZKB_CHECK_CUDA(cudaStreamBeginCapture(s_main, cudaStreamCaptureModeRelaxed));
    const int rc = enqueue(s_main);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s_main, &g);
    ZKB_TRY(rc);
    if (e != cudaSuccess) {
      set_error("graph capture failed: %s", cudaGetErrorString(e));
      return ZKB_ERR_CUDA;
    }
    graph = g;
    ZKB_CHECK_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    size_t nn = 0;
    ZKB_CHECK_CUDA(cudaGraphGetNodes(graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    ZKB_CHECK_CUDA(cudaGraphGetNodes(graph, nodes.data(), &nn));
    kernels_per_run = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType ty;
      ZKB_CHECK_CUDA(cudaGraphNodeGetType(nd, &ty));
      if (ty == cudaGraphNodeTypeKernel) kernels_per_run++;
    }
    return ZKB_OK;
  }

  int run(cudaStream_t s) {
    if (use_graph) {
      if (!exec) ZKB_TRY(capture());
      ZKB_CHECK_CUDA(cudaGraphLaunch(exec, s));
      return ZKB_OK;
    }
    return enqueue(s);
  }

  // ---- autotuning
  // Times fn() on s_main with CUDA events: the best of `reps` after one warm-up.
  template <class Fn>
  int time_ms(Fn fn, int reps, float *best) {
    cudaEvent_t a, b;
    ZKB_CHECK_CUDA(cudaEventCreate(&a));
    ZKB_CHECK_CUDA(cudaEventCreate(&b));
    *best = 1e30f;
    int rc = ZKB_OK;
    for (int r = 0; r <= reps && rc == ZKB_OK; r++) {
      cudaEventRecord(a, s_main);
      rc = fn();
      cudaEventRecord(b, s_main);
      if (rc == ZKB_OK && cudaEventSynchronize(b) != cudaSuccess) rc = ZKB_ERR_CUDA;
      float ms = 0;
      if (rc == ZKB_OK && r > 0 && cudaEventElapsedTime(&ms, a, b) == cudaSuccess) *best = std::min(*best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc == ZKB_ERR_CUDA) set_error("timing run failed: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
  }

  std::string lde_key(size_t i) const {
    char k[96];
    snprintf(k, sizeof k, "lde/%d/%u/%u/%u", spec.field, shapes[i].log_h, shapes[i].width, log_b);
    return k;
  }

  int tune_lde(TuneCache &cache, bool autotune) {
    // the default plans' largest pass (the persistent kernel's tiles take at most 9 bits)
    const int kdef = spec.field == FIELD_BABYBEAR ? (persistent ? 9 : 10) : 7;
    std::vector<std::pair<std::string, LdeTune>> done;
    for (size_t i = 0; i < shapes.size(); i++) {
      const std::string key = lde_key(i);
      bool found = false;
      for (auto &d : done)
        if (d.first == key) {
          tune[i] = d.second;
          found = true;
        }
      if (found) continue;
      if (const std::string *ln = cache.find(key)) {
        long km = 0, cp = 0, cf = 0;
        LdeTune t;
        if (TuneCache::field(*ln, "kmax", &km) && TuneCache::field(*ln, "c_pass", &cp) &&
            TuneCache::field(*ln, "c_fused", &cf)) {
          t.kmax = (int)km;
          t.c_pass = (uint32_t)cp;
          t.c_fused = (uint32_t)cf;
          if (lde_tune_check(spec.field, shapes[i].width, t) == ZKB_OK) {
            tune[i] = t;
            done.emplace_back(key, t);
            tuned_from_cache = true;
            continue;
          }
          clear_error();
        }
      }
      if (!autotune) {
        tune[i] = LdeTune{};
        continue;
      }
      const uint32_t w = shapes[i].width;
      std::vector<LdeTune> cands;
      std::vector<std::vector<int>> seen_plans;
      for (int km = kdef; km >= kdef - 2 && km >= 1; km--) {
        // kernel choices only differ when the pass split does
        std::vector<int> ks;
        const int L = (int)shapes[i].log_h;
        const int np = L > 0 ? (L + km - 1) / km : 0;
        for (int q = 0; q < np; q++) ks.push_back(L / np + (q < L % np ? 1 : 0));
        if (std::find(seen_plans.begin(), seen_plans.end(), ks) != seen_plans.end()) continue;
        seen_plans.push_back(ks);
        for (uint32_t cp : {16u, 8u, 4u})
          for (uint32_t cf : {8u, 4u}) {
            LdeTune t{km, cp, cf};
            if (lde_tune_check(spec.field, w, t) != ZKB_OK) {
              clear_error();
              continue;
            }
            cands.push_back(t);
          }
      }
      if (cands.empty()) cands.push_back(LdeTune{});
      LdeTune best_t = cands[0];
      float best = 1e30f;
      for (const LdeTune &t : cands) {
        float ms = 0;
        ZKB_TRY(time_ms([&] { return lde_one(i, s_main, &t); }, 2, &ms));
        if (ms < best) {
          best = ms;
          best_t = t;
        }
      }
      tune[i] = best_t;
      done.emplace_back(key, best_t);
      char ln[256];
      snprintf(ln, sizeof ln, "{\"key\": \"%s\", \"kmax\": %d, \"c_pass\": %u, \"c_fused\": %u, \"us\": %d}",
               key.c_str(), best_t.kmax, best_t.c_pass, best_t.c_fused, (int)(best * 1000));
      cache.put(key, ln);
    }
    return ZKB_OK;
  }

  std::string batch_key(const char *what) const {
    std::vector<uint32_t> sig;
    for (auto &s : shapes) {
      sig.push_back(s.log_h);
      sig.push_back(s.width);
    }
    const uint64_t h = fnv1a(sig.data(), sig.size() * 4);
    char k[128];
    snprintf(k, sizeof k, "%s/%d/%d/%u/%zu/%016llx", what, spec.field, spec.width, log_b, shapes.size(),
             (unsigned long long)h);
    return k;
  }

  // Persistent form: the Merkle-level fusion (levels above the leaves in the leaf tile,
  // levels per compression tile), timed over whole runs, cached per batch signature.
  int tune_fusion(TuneCache &cache, bool autotune) {
    const std::string key = batch_key("fusion");
    long lv = 0, cv = 0;
    if (const std::string *ln = cache.find(key); ln && TuneCache::field(*ln, "leaf_levels", &lv) &&
                                                 TuneCache::field(*ln, "comp_levels", &cv) && lv >= 0 &&
                                                 lv <= 8 && cv >= 1 && cv <= 8) {
      fusion = MerkleFusion{(uint32_t)lv, (uint32_t)cv};
      tuned_from_cache = true;
      return build_persist();
    }
    if (!autotune) return build_persist();
    float best = 1e30f;
    MerkleFusion bf = fusion;
    for (uint32_t l : {0u, 2u, 4u, 8u})
      for (uint32_t c : {1u, 4u, 8u}) {
        fusion = MerkleFusion{l, c};
        ZKB_TRY(build_persist());
        float ms = 0;
        ZKB_TRY(time_ms([&] { return persist->enqueue(s_main); }, 2, &ms));
        ZKB_TRY(persist->check(s_main));
        if (ms < best) {
          best = ms;
          bf = fusion;
        }
      }
    fusion = bf;
    ZKB_TRY(build_persist());
    char ln[256];
    snprintf(ln, sizeof ln, "{\"key\": \"%s\", \"leaf_levels\": %u, \"comp_levels\": %u, \"us\": %d}",
             key.c_str(), fusion.leaf_levels, fusion.comp_levels, (int)(best * 1000));
    cache.put(key, ln);
    return ZKB_OK;
  }

  int tune_leaf_and_branches(TuneCache &cache, bool autotune, uint32_t fixed_branches) {
    const std::string lk = batch_key("leaf"), bk = batch_key("branches");
    long v = 0;
    if (const std::string *ln = cache.find(lk); ln && TuneCache::field(*ln, "threads", &v) &&
                                                (v == 64 || v == 128 || v == 256)) {
      leaf_threads = (unsigned)v;
      tuned_from_cache = true;
    } else if (autotune) {
      float best = 1e30f;
      for (unsigned th : {64u, 128u, 256u}) {
        float ms = 0;
        ZKB_TRY(time_ms([&] { return hash_dispatch(th, s_main); }, 2, &ms));
        if (ms < best) {
          best = ms;
          leaf_threads = th;
        }
      }
      char ln[256];
      snprintf(ln, sizeof ln, "{\"key\": \"%s\", \"threads\": %u, \"us\": %d}", lk.c_str(), leaf_threads,
               (int)(best * 1000));
      cache.put(lk, ln);
    }
    if (fixed_branches) return assign_branches(fixed_branches);
    if (const std::string *ln = cache.find(bk); ln && TuneCache::field(*ln, "branches", &v) && v >= 1 &&
                                                v <= (long)s_br.size()) {
      ZKB_TRY(assign_branches((uint32_t)v));
      tuned_from_cache = true;
      return ZKB_OK;
    }
    if (!autotune) {
      // default: as many branches as fit, up to four
      for (uint32_t nb = std::min<uint32_t>(4, (uint32_t)s_br.size()); nb >= 1; nb--) {
        if (assign_branches(nb) == ZKB_OK) return ZKB_OK;
        clear_error();
      }
      return assign_branches(1);
    }
    float best = 1e30f;
    uint32_t best_nb = 1;
    for (uint32_t nb : {1u, 2u, 4u, 8u}) {
      if (nb > shapes.size() || nb > s_br.size()) continue;
      if (assign_branches(nb) != ZKB_OK) {  // scratch does not fit: fewer branches only
        clear_error();
        continue;
      }
      if (use_graph) ZKB_TRY(capture());
      float ms = 0;
      ZKB_TRY(time_ms([&] { return run(s_main); }, 2, &ms));
      if (ms < best) {
        best = ms;
        best_nb = nb;
      }
    }
    ZKB_TRY(assign_branches(best_nb));
    char ln[256];
    snprintf(ln, sizeof ln, "{\"key\": \"%s\", \"branches\": %u, \"us\": %d}", bk.c_str(), best_nb,
             (int)(best * 1000));
    cache.put(bk, ln);
    return ZKB_OK;
  }
};

namespace {

constexpr uint32_t MAX_BRANCHES = 8;

int batch_build(zkb_batch *b, const zkb_batch_options &opt) {
  const size_t n = b->shapes.size();
  // the arena is one cudaMalloc: memory the library keeps for reuse goes back first
  ZKB_TRY(release_cached_memory());
  const int OUT = b->out;
  const size_t es = b->es;
  const uint32_t nb_max = std::min<uint32_t>(MAX_BRANCHES, (uint32_t)n);
  // ---- arena layout
  uint64_t off = 0;
  std::vector<uint64_t> in_off(n), lde_off(n), lay_off(n);
  uint64_t total_digests = 0;
  for (size_t i = 0; i < n; i++) {
    const uint64_t rows = 1ull << b->shapes[i].log_h, w = b->shapes[i].width;
    in_off[i] = off;
    off = align256(off + rows * w * es);
    lde_off[i] = off;
    off = align256(off + (rows << b->log_b) * w * es);
  }
  const uint64_t layers_base = off;
  for (size_t i = 0; i < n; i++) {
    lay_off[i] = total_digests;  // digests from layers_base
    total_digests += 2 * b->rows_of(i) - 1;
  }
  off = align256(off + total_digests * OUT * es);
  const uint64_t roots_off = off;
  off = align256(off + n * OUT * es);
  // job tables: n leaf jobs, one compression job per level of every tree, n root offsets
  uint64_t n_comp = 0;
  for (size_t i = 0; i < n; i++) n_comp += b->shapes[i].log_h + b->log_b;
  const uint64_t tables_off = off;
  off = align256(off + n * sizeof(LeafJob) + n_comp * sizeof(CompJob) + n * 8);
  // the same jobs once more as one table set per host group (runs from host memory): the
  // jobs, root offsets and root indices of each group, every group's records 8-byte aligned
  const uint64_t group_tables_off = off;
  const uint64_t group_tables_bytes = n * (sizeof(LeafJob) + 8 + 4 + 8) + n_comp * sizeof(CompJob);
  off = align256(off + group_tables_bytes);
  b->arena_bytes = off;

  size_t free_b = 0, total_b = 0;
  ZKB_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
  ZKB_REQUIRE(b->arena_bytes + (1ull << 30) <= free_b,
              "batch needs %llu bytes of device memory, %llu free", (unsigned long long)b->arena_bytes,
              (unsigned long long)free_b);
  note_device_alloc();
  ZKB_CHECK_CUDA(cudaMalloc(&b->arena, b->arena_bytes));
  char *base = (char *)b->arena;
  b->d_in.resize(n);
  b->d_lde.resize(n);
  b->d_layers.resize(n);
  for (size_t i = 0; i < n; i++) {
    b->d_in[i] = base + in_off[i];
    b->d_lde[i] = base + lde_off[i];
    b->d_layers[i] = base + layers_base + lay_off[i] * OUT * es;
  }
  b->d_roots = base + roots_off;
  if (b->persistent) {
    // Coefficient scratch of the inverse passes in S slots shared round-robin by the traces
    // taken largest first: trace k of that order uses slot k % S after trace k - S, whose
    // fused step (the scratch's last reader) it waits for; the queue runs the traces in
    // rounds of S.  S is as large as free memory allows (2 GiB kept free), at most 16, or
    // at most ZKB_PERSIST_SLOTS when that is set.
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    auto cells = [&](int i) { return (uint64_t)b->shapes[i].width << b->shapes[i].log_h; };
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return cells(x) > cells(y); });
    ZKB_CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
    uint32_t S = 0, s_max = 16;
    if (const char *v = getenv("ZKB_PERSIST_SLOTS"); v && atoi(v) >= 1) s_max = std::min<uint32_t>(16, atoi(v));
    uint64_t coef_total = 0;
    while (S < n && S < s_max) {
      const uint64_t add = align256(cells(ord[S]) * es);
      if (coef_total + add + (2ull << 30) > free_b) break;
      coef_total += add;
      S++;
    }
    ZKB_REQUIRE(S >= 1, "the persistent form needs %llu more bytes of device memory, %llu free",
                (unsigned long long)align256(cells(ord[0]) * es), (unsigned long long)free_b);
    note_device_alloc();
    ZKB_CHECK_CUDA(cudaMalloc(&b->d_coef_all, coef_total));
    std::vector<uint32_t *> slot(S);
    uint64_t o = 0;
    for (uint32_t k = 0; k < S; k++) {
      slot[k] = (uint32_t *)((char *)b->d_coef_all + o);
      o += align256(cells(ord[k]) * es);
    }
    b->coef_slots = S;
    b->coef_of.assign(n, nullptr);
    b->queue_order = ord;
    b->slot_prev.assign(n, -1);
    b->round_of.assign(n, 0);
    for (size_t k = 0; k < n; k++) {
      b->coef_of[ord[k]] = slot[k % S];
      b->slot_prev[k] = k >= S ? (int)(k - S) : -1;
      b->round_of[k] = (int)(k / S);
    }
  }

  // ---- job tables
  std::vector<const void *> data(n);
  std::vector<uint64_t> rows(n), widths(n);
  for (size_t i = 0; i < n; i++) {
    data[i] = b->d_lde[i];
    rows[i] = b->rows_of(i);
    widths[i] = b->shapes[i].width;
  }
  mt::build_tables(data, rows, widths, b->d_layers, b->d_layers[0], OUT, es, &b->joint.t);
  ZKB_REQUIRE(b->joint.t.device_bytes() <= n * sizeof(LeafJob) + n_comp * sizeof(CompJob) + n * 8,
              "internal: batch job tables");
  ZKB_CHECK_CUDA(cudaMemsetAsync(b->arena, 0, layers_base, b->s_main));
  {
    LeafJob *l = nullptr;
    CompJob *c = nullptr;
    uint64_t *r = nullptr;
    ZKB_TRY(mt::upload_tables(b->joint.t, base + tables_off, b->s_main, &l, &c, &r));
    b->joint.leaf = l;
    b->joint.comp = c;
    b->joint.root_off = r;
  }
  // host groups: the copy order puts the small traces at both ends and the largest in
  // the middle (sorted by cells: the even positions ascending, then the odd ones
  // descending); a group closes once it holds `target` cells (1/64 of the batch, at least
  // 2^23) or before a trace that would take it past that; a larger trace forms a group by
  // itself
  std::vector<char> img;
  if (!b->persistent) {
    auto cells = [&](int i) { return (uint64_t)b->shapes[i].width << b->shapes[i].log_h; };
    std::vector<int> sorted(n), ord;
    std::iota(sorted.begin(), sorted.end(), 0);
    std::stable_sort(sorted.begin(), sorted.end(), [&](int x, int y) { return cells(x) < cells(y); });
    for (size_t k = 0; k < n; k += 2) ord.push_back(sorted[k]);
    for (size_t k = (n % 2 ? n - 2 : n - 1); k < n; k -= 2) ord.push_back(sorted[k]);
    uint64_t total = 0;
    for (size_t i = 0; i < n; i++) total += cells((int)i);
    const uint64_t target = std::max<uint64_t>(total / 64, 1ull << 23);
    uint64_t acc = 0;
    std::vector<std::vector<int>> groups(1);
    for (int i : ord) {
      if (!groups.back().empty() && acc + cells(i) > target) {
        groups.emplace_back();
        acc = 0;
      }
      groups.back().push_back(i);
      acc += cells(i);
      if (acc >= target) {
        groups.emplace_back();
        acc = 0;
      }
    }
    if (groups.back().empty()) groups.pop_back();
    img.assign(group_tables_bytes, 0);
    uint64_t to = 0;
    b->host_groups.resize(groups.size());
    for (size_t k = 0; k < groups.size(); k++) {
      HostGroup &g = b->host_groups[k];
      g.traces = groups[k];
      g.member.assign(n, 0);
      const size_t m = g.traces.size();
      std::vector<const void *> gd(m);
      std::vector<uint64_t> gr(m), gw(m);
      std::vector<void *> gl(m);
      std::vector<uint32_t> dst(m);
      for (size_t q = 0; q < m; q++) {
        const int i = g.traces[q];
        g.member[i] = 1;
        gd[q] = data[i];
        gr[q] = rows[i];
        gw[q] = widths[i];
        gl[q] = b->d_layers[i];
        dst[q] = (uint32_t)i;
      }
      mt::build_tables(gd, gr, gw, gl, b->d_layers[0], OUT, es, &g.jobs.t);
      const uint64_t lb = m * sizeof(LeafJob), cb = g.jobs.t.comp.size() * sizeof(CompJob), rb = m * 8,
                     db = (m * 4 + 7) & ~7ull;
      ZKB_REQUIRE(to + lb + cb + rb + db <= group_tables_bytes, "internal: host group job tables");
      char *dev = base + group_tables_off + to;
      memcpy(img.data() + to, g.jobs.t.leaf.data(), lb);
      if (cb) memcpy(img.data() + to + lb, g.jobs.t.comp.data(), cb);
      memcpy(img.data() + to + lb + cb, g.jobs.t.root_off.data(), rb);
      memcpy(img.data() + to + lb + cb + rb, dst.data(), m * 4);
      g.jobs.leaf = (const LeafJob *)dev;
      g.jobs.comp = (const CompJob *)(dev + lb);
      g.jobs.root_off = (const uint64_t *)(dev + lb + cb);
      g.jobs.root_dst = (const uint32_t *)(dev + lb + cb + rb);
      to += lb + cb + rb + db;
    }
    ZKB_CHECK_CUDA(cudaMemcpyAsync(base + group_tables_off, img.data(), to, cudaMemcpyHostToDevice, b->s_main));
  }
  ZKB_TRY(wait_stream(b->s_main));

  // ---- streams and events
  for (uint32_t k = 0; k < nb_max; k++) {
    cudaStream_t s;
    ZKB_CHECK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->s_br.push_back(s);
    cudaEvent_t e;
    ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev_br.push_back(e);
  }
  ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  ZKB_CHECK_CUDA(cudaStreamCreateWithFlags(&b->s_copy, cudaStreamNonBlocking));
  ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&b->ev_host, cudaEventDisableTiming));
  ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&b->ev_copied, cudaEventDisableTiming));
  for (auto &g : b->host_groups) ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&g.copied, cudaEventDisableTiming));

  // ---- tables (built once, outside any capture) and kernel shapes
  b->tune.assign(n, LdeTune{});
  ZKB_TRY(b->assign_branches(1));
  for (size_t i = 0; i < n; i++) ZKB_TRY(b->lde_one(i, b->s_main, nullptr));
  ZKB_TRY(wait_stream(b->s_main));
  TuneCache cache;
  if (opt.tune_cache) cache.path = opt.tune_cache;
  cache.load();
  cudaEvent_t t0, t1;
  ZKB_CHECK_CUDA(cudaEventCreate(&t0));
  ZKB_CHECK_CUDA(cudaEventCreate(&t1));
  cudaEventRecord(t0, b->s_main);
  int rc = b->tune_lde(cache, opt.autotune != 0);
  // one LDE of every trace with its final kernel shapes builds every table those shapes
  // read (some depend on the pass split), so nothing is built inside a graph capture
  for (size_t i = 0; i < n && rc == ZKB_OK; i++) rc = b->lde_one(i, b->s_main, &b->tune[i]);
  if (rc == ZKB_OK) rc = wait_stream(b->s_main);
  if (rc == ZKB_OK)
    rc = b->persistent ? b->tune_fusion(cache, opt.autotune != 0)
                       : b->tune_leaf_and_branches(cache, opt.autotune != 0, std::min(opt.branches, nb_max));
  cudaEventRecord(t1, b->s_main);
  cudaEventSynchronize(t1);
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  b->tune_ms = ms;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  ZKB_TRY(rc);
  if (opt.autotune) cache.save();
  if (b->use_graph) ZKB_TRY(b->capture());


  // ---- borrowed per-trace trees for openings
  for (size_t i = 0; i < n; i++) {
    auto t = std::make_unique<zkb_tree>();
    DeviceTree &d = t->t;
    d.spec = b->spec;
    d.device = b->device;
    d.stream = b->s_main;
    d.d_layers = b->d_layers[i];
    d.borrowed = true;
    uint64_t o = 0;
    for (uint64_t len : b->joint.t.layer_len[i]) {
      d.layer_off.push_back(o);
      d.layer_len.push_back(len);
      o += len;
    }
    d.mats.push_back(TreeMatrix{b->d_lde[i], b->rows_of(i), b->shapes[i].width});
    b->trees.push_back(std::move(t));
  }
  return ZKB_OK;
}

}  // namespace

extern "C" {

int zkb_batch_create(const zkb_hasher *hasher, const zkb_batch_shape *shapes, size_t n,
                     const zkb_batch_options *opt, zkb_batch **out) {
  clear_error();
  ZKB_REQUIRE(hasher && shapes && opt && out, "null arguments");
  ZKB_TRY(library_gate());
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device available");
    return ZKB_DECLINED;
  }
  ZKB_REQUIRE(n >= 1 && n <= (size_t)MAX_BATCH, "batch of %zu traces (1..%d)", n, MAX_BATCH);
  auto b = std::make_unique<zkb_batch>();
  ZKB_CHECK_CUDA(cudaGetDevice(&b->device));
  if (!make_hasher_spec(hasher->field, (int)hasher->width, hasher->seed, &b->spec)) {
    set_error("unsupported Poseidon2 hasher: field %d width %u", hasher->field, hasher->width);
    return ZKB_ERR_UNSUPPORTED;
  }
  const int two_adicity = hasher->field == ZKB_FIELD_BABYBEAR ? 27 : 32;
  ZKB_REQUIRE(opt->log_blowup >= 1 && opt->log_blowup <= 4, "log_blowup must be in [1, 4]");
  for (size_t i = 0; i < n; i++)
    ZKB_REQUIRE(shapes[i].width >= 1 && shapes[i].width <= 4096 &&
                    (int)(shapes[i].log_h + opt->log_blowup) <= two_adicity && shapes[i].log_h <= 26,
                "trace %zu: unsupported shape 2^%u x %u", i, shapes[i].log_h, shapes[i].width);
  b->shapes.assign(shapes, shapes + n);
  b->log_b = opt->log_blowup;
  b->es = field_elem_bytes(hasher->field);
  b->out = b->spec.out;
  b->use_graph = opt->use_graph != 0;
  b->persistent = opt->use_graph == 2;
  if (b->persistent) {
    ZKB_REQUIRE(hasher->field == ZKB_FIELD_BABYBEAR && hasher->width == 16,
                "the persistent form commits BabyBear traces with the width-16 hasher");
    for (size_t i = 0; i < n; i++)
      ZKB_REQUIRE(shapes[i].width % 8 == 0 && shapes[i].log_h >= 1 && shapes[i].log_h + opt->log_blowup <= 25,
                  "trace %zu: the persistent form takes widths that are multiples of 8 and 2^1..2^%u rows (got "
                  "2^%u x %u)",
                  i, 25 - opt->log_blowup, shapes[i].log_h, shapes[i].width);
  }
  bool ok;
  if (b->spec.field == FIELD_BABYBEAR)
    ok = build_p2_params<BabyBear, 16>(b->spec, &b->p_bb16);
  else if (b->spec.width == 16)
    ok = build_p2_params<Goldilocks, 16>(b->spec, &b->p_gl16);
  else
    ok = build_p2_params<Goldilocks, 12>(b->spec, &b->p_gl12);
  ZKB_REQUIRE(ok, "invalid Poseidon2 parameters");
  ZKB_CHECK_CUDA(cudaStreamCreateWithFlags(&b->s_main, cudaStreamNonBlocking));
  ZKB_TRY(batch_build(b.get(), *opt));
  *out = b.release();
  return ZKB_OK;
}

int zkb_batch_trace_ptr(zkb_batch *b, size_t i, void **d_trace) {
  clear_error();
  ZKB_REQUIRE(b && d_trace && i < b->shapes.size(), "invalid trace request");
  *d_trace = b->d_in[i];
  return ZKB_OK;
}

int zkb_batch_copy_in(zkb_batch *b, size_t i, const void *src, int src_on_device, void *stream) {
  clear_error();
  ZKB_REQUIRE(b && src && i < b->shapes.size(), "invalid copy request");
  ZKB_CHECK_CUDA(cudaSetDevice(b->device));
  const uint64_t bytes = (1ull << b->shapes[i].log_h) * b->shapes[i].width * b->es;
  ZKB_CHECK_CUDA(cudaMemcpyAsync(b->d_in[i], src, bytes,
                                 src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 resolve_stream(stream)));
  return ZKB_OK;
}

int zkb_batch_run(zkb_batch *b, void *stream) {
  clear_error();
  ZKB_REQUIRE(b != nullptr, "null batch");
  ZKB_TRY(library_gate());
  ZKB_CHECK_CUDA(cudaSetDevice(b->device));
  return b->run(resolve_stream(stream));
}

int zkb_batch_run_host(zkb_batch *b, const void *const *traces, void *stream) {
  clear_error();
  ZKB_REQUIRE(b && traces, "null arguments");
  ZKB_TRY(library_gate());
  ZKB_CHECK_CUDA(cudaSetDevice(b->device));
  return b->run_host(traces, resolve_stream(stream));
}

int zkb_batch_roots(zkb_batch *b, void *roots_out, void *stream) {
  clear_error();
  ZKB_REQUIRE(b && roots_out, "null arguments");
  ZKB_CHECK_CUDA(cudaSetDevice(b->device));
  cudaStream_t s = resolve_stream(stream);
  if (b->persistent) ZKB_TRY(b->persist->check(s));  // a work item's wait gave up: no roots
  ZKB_CHECK_CUDA(cudaMemcpyAsync(roots_out, b->d_roots, b->shapes.size() * b->out * b->es,
                                 cudaMemcpyDeviceToHost, s));
  ZKB_TRY(wait_stream(s));
  return ZKB_OK;
}

int zkb_batch_tree(zkb_batch *b, size_t i, const zkb_tree **tree) {
  clear_error();
  ZKB_REQUIRE(b && tree && i < b->trees.size(), "invalid tree request");
  *tree = b->trees[i].get();
  return ZKB_OK;
}

int zkb_batch_info(const zkb_batch *b, zkb_batch_info_t *info) {
  clear_error();
  ZKB_REQUIRE(b && info, "null arguments");
  info->device_bytes = b->arena_bytes;
  info->kernels_per_run = b->use_graph ? b->kernels_per_run : 0;
  info->branches = b->persistent ? 0 : b->branches;
  info->leaf_threads = b->leaf_threads;
  info->use_graph = b->persistent ? 2 : b->use_graph ? 1 : 0;
  info->tuned_from_cache = b->tuned_from_cache ? 1 : 0;
  info->tune_ms = b->tune_ms;
  return ZKB_OK;
}

int zkb_batch_lde_tune(const zkb_batch *b, size_t i, int *kmax, uint32_t *c_pass, uint32_t *c_fused) {
  clear_error();
  ZKB_REQUIRE(b && i < b->tune.size() && kmax && c_pass && c_fused, "invalid request");
  *kmax = b->tune[i].kmax;
  *c_pass = b->tune[i].c_pass;
  *c_fused = b->tune[i].c_fused;
  return ZKB_OK;
}

int zkb_batch_set_merkle_fusion(zkb_batch *b, uint32_t leaf_levels, uint32_t comp_levels) {
  clear_error();
  ZKB_REQUIRE(b != nullptr, "null batch");
  ZKB_REQUIRE(b->persistent, "Merkle-level fusion applies to the persistent form (use_graph = 2)");
  ZKB_REQUIRE(leaf_levels <= 8 && comp_levels >= 1 && comp_levels <= 8,
              "leaf levels %u (0..8), compression levels %u (1..8)", leaf_levels, comp_levels);
  ZKB_CHECK_CUDA(cudaSetDevice(b->device));
  ZKB_TRY(wait_stream(b->s_main));
  b->fusion = MerkleFusion{leaf_levels, comp_levels};
  ZKB_TRY(b->build_persist());
  if (b->use_graph) ZKB_TRY(b->capture());
  return ZKB_OK;
}

int zkb_batch_queue_info(const zkb_batch *b, zkb_batch_queue_info_t *info) {
  clear_error();
  ZKB_REQUIRE(b && info, "null arguments");
  ZKB_REQUIRE(b->persistent && b->persist, "not a persistent plan");
  const PersistStats st = b->persist->stats();
  info->items = st.items;
  info->steps = st.steps;
  info->stages = st.stages;
  info->grid = st.grid;
  info->leaf_levels = b->fusion.leaf_levels;
  info->comp_levels = b->fusion.comp_levels;
  return ZKB_OK;
}

int zkb_batch_profile(zkb_batch *b, void *stream, double *busy_ms, double *span_ms) {
  clear_error();
  ZKB_REQUIRE(b && busy_ms && span_ms, "null arguments");
  ZKB_REQUIRE(b->persistent && b->persist, "not a persistent plan");
  ZKB_CHECK_CUDA(cudaSetDevice(b->device));
  return b->persist->profile(resolve_stream(stream), busy_ms, span_ms);
}

int zkb_debug_batch_stalled_run(zkb_batch *b, uint64_t spin_limit, void *stream) {
  clear_error();
  ZKB_REQUIRE(b != nullptr, "null batch");
  ZKB_REQUIRE(b->persistent && b->persist, "not a persistent plan");
  ZKB_REQUIRE(spin_limit >= 1 && spin_limit <= (1ull << 24), "spin limit %llu (1..2^24)",
              (unsigned long long)spin_limit);
  ZKB_CHECK_CUDA(cudaSetDevice(b->device));
  return b->persist->enqueue_stalled(resolve_stream(stream), spin_limit);
}

void zkb_batch_free(zkb_batch *b) { delete b; }

}  // extern "C"
