// persist.cu — a batch of BabyBear traces committed by ONE persistent kernel.
//
// The plan cuts every trace's commitment into steps — the NTT passes of its coset LDE
// (inverse passes, the fused middle, forward passes), the leaf hashing, the compression
// levels — and every step into items (ranges of CTA-tiles).  The items of all traces form
// one queue in a dependency-respecting order (wavefront: step k of every trace, largest
// first, then step k+1).  Each block of the kernel claims the next item with an atomic
// increment, waits until every item of the step it depends on has finished (a counter per
// step), runs the item's tiles and bumps its own step's counter.  Items only depend on
// items earlier in the queue, each held by a running block, so the queue always drains;
// no grid-wide barrier is used and the blocks need not be co-resident.  While one trace
// waits between two of its steps, the blocks take the other traces' items, and the small
// traces' kernels no longer sit in their own launches at a fraction of the GPU.
//
// Every wait is bounded: a block polls its counter at most `spin_limit` times, then
// records the item in an error word, and every block leaves the queue once the word is
// set; the host reads the word after the run and reports ZKB_ERR_TIMEOUT.
//
// The tiles are the standalone kernels' own code (ntt_tile.cuh, poseidon2.cuh), so every
// root equals the plain per-trace commitment (TwoAdicFriPcs::commit over one matrix,
// vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:84-151).  Data written by other blocks of
// the same launch is read after the counter's acquire: the NTT tiles read through L2
// (ld.global.cg; the forward passes rewrite in place what earlier passes read), while the
// leaf and compression tiles read through L1 — nothing in a run loads the final LDE or a
// digest layer before it is written (L1 starts empty at every launch), and the leaf
// hash's 32-byte reads of one row share its lines.
// Merkle-level fusion: a leaf tile of 256 rows can also compress its digests up to
// `leaf_levels` levels in shared memory, and a compression tile computes `comp_levels`
// levels; the batch plan's autotuner chooses both.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.cuh"
#include "ntt_tile.cuh"
#include "persist.cuh"
#include "poseidon2.cuh"

namespace zkb {
namespace {

constexpr int PT = 256;        // threads per block
constexpr int MAX_K = 9;       // largest pass: 16 columns x 2^(9/2) rows of threads = 256
constexpr uint32_t NONE = 0xffffffffu;
// Polls before a wait gives up in a normal run: tens of seconds (256 ns sleeps), well above
// the longest legitimate wait (a block can wait for several steps of the largest trace).
constexpr uint64_t SPIN_LIMIT = 32ull << 20;

enum : uint8_t { PASS = 0, FUSED = 1, LEAF = 2, COMP = 3 };

struct Stage {
  uint8_t kind;
  uint8_t K;          // pass / fused: bits
  uint8_t C;          // pass / fused: columns per tile
  uint8_t levels;     // leaf: levels above the leaves in the tile; comp: levels per tile
  uint8_t inverse;    // pass: inverse transform
  uint8_t pad[3];
  uint32_t step;      // counter bumped by this stage's items
  uint32_t dep;       // counter waited for (NONE: none)
  uint32_t dep_target;
  uint32_t tile_rows; // leaf: rows per tile; comp: outputs of the first level per tile
  PassGeom pg;
  FusedGeom fg;
  const uint32_t *in;   // pass / fused input; leaf: LDE rows; comp: the layer below
  uint32_t *out;        // pass / fused output; leaf: leaf digests; comp: the first layer made
  const uint32_t *t0, *t1, *t2, *t3;  // pass: twiddles; fused: itw, ftw, ctab_t, ftw_t
  // the register DIFs' w_64 tables (inverse, forward) in device memory: read through the
  // stage, they are not loop-invariant to the compiler, which would otherwise hoist all
  // 128 words out of the block's item loop and spill them
  const SmallTw<BabyBear> *sti, *stf;
  uint64_t rows;        // leaf: LDE rows; comp: nodes of the first layer made
  uint32_t width;       // leaf: row width (multiple of 8)
  uint32_t *root;       // set on the stage that makes the top level
};

struct Item {
  uint32_t stage, tile0, ntiles;
};

struct Params {
  const Stage *stages;
  const Item *items;
  uint32_t n_items;
  uint32_t *counters;   // per step, then the queue head, then the error word
  uint64_t spin_limit;
  uint64_t *prof;       // profiled runs: per item, the global timer at its start and end
  P2Params<BabyBear, 16> p2;
};

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The NTT tiles of one item, one function per kernel shape: not inlined, so each gets its
// own register allocation (inlined into one loop they spilled), and each names the
// dynamic shared memory itself, so its accesses stay shared-space loads and stores.
template <int K, int C>
__device__ __noinline__ void pass_item(const Stage *st, uint32_t tile0, uint32_t ntiles) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmallTw<BabyBear> &stw = st->inverse ? *st->sti : *st->stf;
  for (uint32_t t = 0; t < ntiles; t++) {
    ntt_pass_tile<BabyBear, (K + 1) / 2, K / 2, C, true>(st->in, st->out, st->pg, st->t0, 0u, stw, tile0 + t,
                                                          smem);
    __syncthreads();  // shared memory is reused by the next tile
  }
}

template <int K, int C>
__device__ __noinline__ void fused_item(const Stage *st, uint32_t tile0, uint32_t ntiles) {
  extern __shared__ __align__(16) unsigned char smem[];
  for (uint32_t t = 0; t < ntiles; t++) {
    lde_fused_tile<BabyBear, (K + 1) / 2, K / 2, C, true>(st->in, st->out, st->fg, st->t0, st->t1, st->t2, st->t3,
                                                           *st->sti, *st->stf, tile0 + t, smem);
    __syncthreads();
  }
}

// Column chunks of the NTT tiles: as many columns as fill the block (C << (K / 2) = 256
// threads, at most 64 columns), narrower chunks (32, 16, 8) for what the width leaves.
__host__ __device__ constexpr uint32_t c_full(int K) {
  return (256u >> (K / 2)) > 64u ? 64u : (256u >> (K / 2));
}

template <int K>
__device__ __forceinline__ void pass_k(const Stage *st, uint32_t tile0, uint32_t ntiles) {
  switch (st->C) {
    case 8: pass_item<K, 8>(st, tile0, ntiles); break;
    case 16: pass_item<K, 16>(st, tile0, ntiles); break;
    case 32:
      if constexpr (c_full(K) >= 32) pass_item<K, 32>(st, tile0, ntiles);
      break;
    case 64:
      if constexpr (c_full(K) >= 64) pass_item<K, 64>(st, tile0, ntiles);
      break;
    default: break;
  }
}

template <int K>
__device__ __forceinline__ void fused_k(const Stage *st, uint32_t tile0, uint32_t ntiles) {
  switch (st->C) {
    case 8: fused_item<K, 8>(st, tile0, ntiles); break;
    case 16:
      if constexpr (c_full(K) >= 16) fused_item<K, 16>(st, tile0, ntiles);
      break;
    case 32:
      if constexpr (c_full(K) >= 32) fused_item<K, 32>(st, tile0, ntiles);
      break;
    case 64:
      if constexpr (c_full(K) >= 64) fused_item<K, 64>(st, tile0, ntiles);
      break;
    default: break;
  }
}

__device__ __forceinline__ void pass_dispatch(const Stage *st, uint32_t tile0, uint32_t ntiles) {
  switch (st->K) {
    case 1: pass_k<1>(st, tile0, ntiles); break;
    case 2: pass_k<2>(st, tile0, ntiles); break;
    case 3: pass_k<3>(st, tile0, ntiles); break;
    case 4: pass_k<4>(st, tile0, ntiles); break;
    case 5: pass_k<5>(st, tile0, ntiles); break;
    case 6: pass_k<6>(st, tile0, ntiles); break;
    case 7: pass_k<7>(st, tile0, ntiles); break;
    case 8: pass_k<8>(st, tile0, ntiles); break;
    case 9: pass_k<9>(st, tile0, ntiles); break;
    default: break;
  }
}

__device__ __forceinline__ void fused_dispatch(const Stage *st, uint32_t tile0, uint32_t ntiles) {
  switch (st->K) {
    case 1: fused_k<1>(st, tile0, ntiles); break;
    case 2: fused_k<2>(st, tile0, ntiles); break;
    case 3: fused_k<3>(st, tile0, ntiles); break;
    case 4: fused_k<4>(st, tile0, ntiles); break;
    case 5: fused_k<5>(st, tile0, ntiles); break;
    case 6: fused_k<6>(st, tile0, ntiles); break;
    case 7: fused_k<7>(st, tile0, ntiles); break;
    case 8: fused_k<8>(st, tile0, ntiles); break;
    case 9: fused_k<9>(st, tile0, ntiles); break;
    default: break;
  }
}

// Levels above n0 digests held in sm (internal domain, tile `tile` of their level):
// level f has n0 >> f nodes, written to `layer` (the first level above, len_below / 2
// nodes) and on; the node that is the tree's root also goes to `root`.
__device__ __forceinline__ void merkle_up(uint32_t tile, uint32_t n0, int levels, uint32_t *layer,
                                          uint64_t len_below, uint32_t *root, const Params &p, uint32_t *sm) {
  using D = Dom<BabyBear>;
  uint64_t len = len_below;
  for (int f = 1; f <= levels; f++) {
    const uint32_t n = n0 >> f;
    len >>= 1;
    uint32_t s[16];
    __syncthreads();  // the level below is in sm
    if (threadIdx.x < n) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        s[k] = sm[(2 * threadIdx.x) * 8 + k];
        s[8 + k] = sm[(2 * threadIdx.x + 1) * 8 + k];
      }
    }
    __syncthreads();  // every child read before any parent overwrites sm
    if (threadIdx.x < n) {
      p2_permute<BabyBear, 16>(s, p.p2);
      uint32_t *o = layer + ((uint64_t)tile * n + threadIdx.x) * 8;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        sm[threadIdx.x * 8 + k] = s[k];
        o[k] = D::leave(s[k]);
      }
      if (len == 1 && root) {
#pragma unroll
        for (int k = 0; k < 8; k++) root[k] = D::leave(s[k]);
      }
    }
    layer += len * 8;
  }
}

// Leaf digests of tile_rows rows (PaddingFreeSponge<16, 8, 8>, widths a multiple of 8),
// then `levels` levels above them.
__device__ __forceinline__ void leaf_tile(const Stage &st, uint32_t tile, const Params &p, uint32_t *sm) {
  using D = Dom<BabyBear>;
  const uint32_t TR = st.tile_rows;
  if (threadIdx.x < TR) {
    const uint64_t row = (uint64_t)tile * TR + threadIdx.x;
    uint32_t s[16];
#pragma unroll
    for (int i = 0; i < 16; i++) s[i] = 0;
    const uint32_t *rp = st.in + row * st.width;
    for (uint32_t c = 0; c < st.width; c += 8) {
#pragma unroll
      for (int i = 0; i < 8; i++) s[i] = D::enter(rp[c + i]);
      p2_permute<BabyBear, 16>(s, p.p2);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) st.out[row * 8 + k] = D::leave(s[k]);
    if (st.levels) {
#pragma unroll
      for (int k = 0; k < 8; k++) sm[threadIdx.x * 8 + k] = s[k];
    }
  }
  if (st.levels) merkle_up(tile, TR, st.levels, st.out + st.rows * 8, st.rows, st.root, p, sm);
}

// tile_rows nodes of one level from their children in the level below, then levels - 1
// levels above them.
__device__ __forceinline__ void comp_tile(const Stage &st, uint32_t tile, const Params &p, uint32_t *sm) {
  using D = Dom<BabyBear>;
  const uint32_t TN = st.tile_rows;
  if (threadIdx.x < TN) {
    const uint64_t i = (uint64_t)tile * TN + threadIdx.x;
    uint32_t s[16];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      s[k] = D::enter(st.in[(2 * i) * 8 + k]);
      s[8 + k] = D::enter(st.in[(2 * i + 1) * 8 + k]);
    }
    p2_permute<BabyBear, 16>(s, p.p2);
#pragma unroll
    for (int k = 0; k < 8; k++) {
      st.out[i * 8 + k] = D::leave(s[k]);
      sm[threadIdx.x * 8 + k] = s[k];
    }
    if (st.rows == 1 && st.root) {
#pragma unroll
      for (int k = 0; k < 8; k++) st.root[k] = D::leave(s[k]);
    }
  }
  merkle_up(tile, TN, st.levels - 1, st.out + st.rows * 8, st.rows, st.root, p, sm);
}

__global__ void __launch_bounds__(PT, 4) persist_kernel(const __grid_constant__ Params p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ uint32_t s_item;
  for (;;) {
    if (threadIdx.x == 0) {
      uint32_t *q_head = p.counters - 2;   // head and error sit just before the step counters
      uint32_t *q_err = p.counters - 1;
      uint32_t it = NONE;
      if (ld_acquire(q_err) == 0) {
        it = atomicAdd(q_head, 1u);
        if (it >= p.n_items) {
          it = NONE;
        } else {
          const Stage &st = p.stages[p.items[it].stage];
          if (st.dep != NONE) {
            uint64_t spins = 0;
            while (ld_acquire(p.counters + st.dep) < st.dep_target) {
              if (ld_acquire(q_err) != 0) {
                it = NONE;
                break;
              }
              if (++spins > p.spin_limit) {
                atomicCAS(q_err, 0u, it + 1);
                it = NONE;
                break;
              }
              __nanosleep(256);
            }
          }
        }
      }
      s_item = it;
    }
    __syncthreads();
    const uint32_t it = s_item;
    if (it == NONE) return;
    const Item item = p.items[it];
    const Stage &st = p.stages[item.stage];
    if (p.prof && threadIdx.x == 0) p.prof[2 * it] = global_ns();
    if (st.kind == PASS) {
      pass_dispatch(&st, item.tile0, item.ntiles);
    } else if (st.kind == FUSED) {
      fused_dispatch(&st, item.tile0, item.ntiles);
    } else if (st.kind == LEAF && st.levels == 0) {
      // no shared memory: the warps run through the item's rows independently
      for (uint32_t t = 0; t < item.ntiles; t++) leaf_tile(st, item.tile0 + t, p, nullptr);
    } else {
      for (uint32_t t = 0; t < item.ntiles; t++) {
        if (st.kind == LEAF)
          leaf_tile(st, item.tile0 + t, p, reinterpret_cast<uint32_t *>(smem));
        else
          comp_tile(st, item.tile0 + t, p, reinterpret_cast<uint32_t *>(smem));
        __syncthreads();  // shared memory is reused by the next tile
      }
    }
    __syncthreads();  // every thread has read s_item before the next claim
    if (p.prof && threadIdx.x == 0) p.prof[2 * it + 1] = global_ns();
    if (threadIdx.x == 0) {
      __threadfence();  // the item's writes before its count
      atomicAdd(p.counters + st.step, 1u);
    }
  }
}

template <int K>
constexpr size_t max_tile_smem() {
  if constexpr (K == 0) {
    return (size_t)PT * 8 * 4;  // leaf / compression: 256 digests
  } else {
    constexpr uint32_t CF = c_full(K);
    constexpr size_t a = pass_tile_smem<BabyBear, (K + 1) / 2, K / 2, CF>();
    constexpr size_t b = pass_tile_smem<BabyBear, (K + 1) / 2, K / 2, 8>();
    constexpr size_t c = fused_tile_smem<BabyBear, (K + 1) / 2, K / 2, CF>();
    constexpr size_t d = fused_tile_smem<BabyBear, (K + 1) / 2, K / 2, 8>();
    constexpr size_t ab = a > b ? a : b, cd = c > d ? c : d;
    constexpr size_t m = ab > cd ? ab : cd;
    constexpr size_t r = max_tile_smem<K - 1>();
    return m > r ? m : r;
  }
}

uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }

int ilog2(uint64_t x) {
  int l = 0;
  while ((1ull << l) < x) l++;
  return l;
}

}  // namespace

PersistPlan::~PersistPlan() {
  if (d_ || d_prof_) {
    cudaSetDevice(device_);
    if (d_) cudaFree(d_);
    if (d_prof_) cudaFree(d_prof_);
  }
}

int PersistPlan::build(const std::vector<PersistTrace> &traces, int log_b, const P2Params<BabyBear, 16> &p2,
                       const MerkleFusion &fusion, cudaStream_t s) {
  ZKB_REQUIRE(!traces.empty(), "empty persistent plan");
  ZKB_REQUIRE(fusion.leaf_levels <= 8 && fusion.comp_levels >= 1 && fusion.comp_levels <= 8,
              "Merkle fusion: leaf levels %u (0..8), compression levels %u (1..8)", fusion.leaf_levels,
              fusion.comp_levels);
  ZKB_CHECK_CUDA(cudaGetDevice(&device_));
  int sms = 0;
  ZKB_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
  smem_ = max_tile_smem<MAX_K>();
  ZKB_CHECK_CUDA(cudaFuncSetAttribute(persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_));
  int per_sm = 0;
  ZKB_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persist_kernel, PT, smem_));
  ZKB_REQUIRE(per_sm >= 1, "the persistent kernel does not fit on an SM");
  const uint32_t resident = (uint32_t)(per_sm * sms);
  // items per stage: enough for every block to take a few, so a step's tail is short
  const uint64_t target_items = 4ull * resident;

  std::vector<Stage> stages;
  std::vector<std::vector<uint32_t>> step_stages;  // per step: its stages
  std::vector<std::vector<uint32_t>> trace_steps(traces.size());
  std::vector<uint32_t> fused_step(traces.size(), NONE);
  for (size_t t = 0; t < traces.size(); t++)
    ZKB_REQUIRE(traces[t].slot_prev < (int)t && traces[t].round >= 0 &&
                    (traces[t].slot_prev < 0 || traces[traces[t].slot_prev].round < traces[t].round),
                "internal: trace %zu scratch order", t);
  std::vector<uint64_t> tiles_of;
  auto new_step = [&](size_t t) {
    step_stages.emplace_back();
    trace_steps[t].push_back((uint32_t)(step_stages.size() - 1));
    return (uint32_t)(step_stages.size() - 1);
  };
  auto add_stage = [&](const Stage &st, uint64_t tiles) {
    ZKB_REQUIRE(tiles >= 1 && tiles < (1ull << 32), "internal: %llu tiles in one stage", (unsigned long long)tiles);
    stages.push_back(st);
    tiles_of.push_back(tiles);
    step_stages[st.step].push_back((uint32_t)(stages.size() - 1));
    return ZKB_OK;
  };

  for (size_t t = 0; t < traces.size(); t++) {
    const PersistTrace &tr = traces[t];
    const int L = tr.log_h;
    const uint32_t w = tr.width;
    ZKB_REQUIRE(w >= 8 && w % 8 == 0, "trace %zu: the persistent form takes widths that are multiples of 8 (%u)",
                t, w);
    ZKB_REQUIRE(L >= 1 && L + log_b <= 25, "trace %zu: 2^%d rows (1..2^%d in the persistent form)", t, L,
                25 - log_b);
    LdePlanBB lp;
    ZKB_TRY(lde_plan_babybear(L, log_b, std::min(std::max(tr.kmax, 1), MAX_K), &lp, s));
    const std::vector<int> &ks = lp.ks;
    // the first step waits until the scratch's previous user has read it for the last time
    uint32_t prev = tr.slot_prev >= 0 ? fused_step[tr.slot_prev] : NONE;
    // column segments of a pass: 16 columns per tile for the bulk, 8 for a remainder
    // column segments: the widest chunk that fills the block for this pass size, then
    // narrower ones for what is left of the width (a multiple of 8)
    auto segments = [&](int K) {
      std::vector<std::pair<uint32_t, uint32_t>> v;  // (first column, chunk)
      uint32_t c0 = 0;
      for (uint32_t C = c_full(K); C >= 8; C /= 2)
        for (; c0 + C <= w; c0 += C) v.emplace_back(c0, C);
      return v;
    };
    auto pass_step = [&](const uint32_t *src, uint32_t *dst, int K, int lo, bool inverse, uint64_t n_blocks,
                         const uint32_t *tw) -> int {
      const uint32_t step = new_step(t);
      std::vector<std::pair<uint32_t, uint32_t>> seg = segments(K);
      for (size_t q = 0; q < seg.size();) {
        // consecutive chunks of one width form one stage
        const uint32_t c0 = seg[q].first, C = seg[q].second;
        uint32_t cols = 0;
        while (q < seg.size() && seg[q].second == C) {
          cols += C;
          q++;
        }
        Stage st{};
        st.kind = PASS;
        st.K = (uint8_t)K;
        st.C = (uint8_t)C;
        st.inverse = inverse;
        st.step = step;
        st.dep = prev;
        st.pg.L = L;
        st.pg.lo = lo;
        st.pg.width = w;
        st.pg.chunks_per_row = cols / C;
        st.pg.groups = 1u << (L - K);
        st.pg.block_stride = (uint64_t)w << L;
        st.pg.twist = lo > 0;
        st.in = src + c0;
        st.out = dst + c0;
        st.t0 = tw;
        ZKB_TRY(add_stage(st, (uint64_t)st.pg.chunks_per_row * st.pg.groups * n_blocks));
      }
      prev = step;
      return ZKB_OK;
    };
    // inverse passes over all but the lowest bits: input -> coefficient scratch
    int hi = L;
    for (size_t i = 0; i + 1 < ks.size(); i++) {
      ZKB_TRY(pass_step(i == 0 ? tr.in : tr.coef, tr.coef, ks[i], hi - ks[i], true, 1, lp.itw));
      hi -= ks[i];
    }
    // fused middle: last inverse pass, coset twists, first forward pass of every coset
    {
      const int Kf = ks.back();
      const uint32_t step = new_step(t);
      std::vector<std::pair<uint32_t, uint32_t>> seg = segments(Kf);
      for (size_t q = 0; q < seg.size();) {
        const uint32_t c0 = seg[q].first, C = seg[q].second;
        uint32_t cols = 0;
        while (q < seg.size() && seg[q].second == C) {
          cols += C;
          q++;
        }
        Stage st{};
        st.kind = FUSED;
        st.K = (uint8_t)Kf;
        st.C = (uint8_t)C;
        st.step = step;
        st.dep = prev;
        st.fg.L = L;
        st.fg.width = w;
        st.fg.chunks_per_row = cols / C;
        st.fg.blocks = 1u << (L - Kf);
        st.fg.log_b = log_b;
        st.fg.n = 1ull << L;
        st.in = (ks.size() > 1 ? tr.coef : tr.in) + c0;
        st.out = tr.lde + c0;
        st.t0 = lp.itw;
        st.t1 = lp.ftw;
        st.t2 = lp.ctab_t;
        st.t3 = lp.ftw_t;
        ZKB_TRY(add_stage(st, (uint64_t)st.fg.chunks_per_row * st.fg.blocks));
      }
      prev = step;
      fused_step[t] = step;
    }
    // remaining forward passes, in place on the coset blocks
    hi = L - ks.back();
    for (int i = (int)ks.size() - 2; i >= 0; i--) {
      ZKB_TRY(pass_step(tr.lde, tr.lde, ks[i], hi - ks[i], false, 1ull << log_b, lp.ftw));
      hi -= ks[i];
    }
    // leaf hashing, then the compression levels
    const uint64_t rows = 1ull << (L + log_b);
    const int depth = L + log_b;  // levels above the leaves
    uint64_t lay_off = 0;         // digests from the leaves to the current layer
    {
      const uint32_t step = new_step(t);
      Stage st{};
      st.kind = LEAF;
      st.step = step;
      st.dep = prev;
      st.tile_rows = (uint32_t)std::min<uint64_t>(PT, rows);
      st.levels = (uint8_t)std::min<int>((int)fusion.leaf_levels, ilog2(st.tile_rows));
      st.in = tr.lde;
      st.out = tr.layers;
      st.rows = rows;
      st.width = w;
      st.root = st.levels == depth ? tr.root : nullptr;
      ZKB_TRY(add_stage(st, rows / st.tile_rows));
      prev = step;
      // layers made so far: the leaves and st.levels above them
      int made = st.levels;
      uint64_t len = rows;
      lay_off = 0;
      for (int f = 0; f < made; f++) {
        lay_off += len;
        len >>= 1;
      }
      // len: nodes of the last layer made; lay_off: its offset
      while (made < depth) {
        const uint64_t next = len >> 1;
        const uint32_t cstep = new_step(t);
        Stage c{};
        c.kind = COMP;
        c.step = cstep;
        c.dep = prev;
        c.tile_rows = (uint32_t)std::min<uint64_t>(PT, next);
        c.levels = (uint8_t)std::min<int>({(int)fusion.comp_levels, ilog2(c.tile_rows) + 1, depth - made});
        c.in = tr.layers + lay_off * 8;
        c.out = tr.layers + (lay_off + len) * 8;
        c.rows = next;
        c.root = made + c.levels == depth ? tr.root : nullptr;
        ZKB_TRY(add_stage(c, next / c.tile_rows));
        prev = cstep;
        for (int f = 0; f < c.levels; f++) {
          lay_off += len;
          len >>= 1;
        }
        made += c.levels;
      }
    }
  }

  // ---- items: each stage cut into ranges of tiles
  const uint32_t n_steps = (uint32_t)step_stages.size();
  std::vector<uint32_t> stage_items(stages.size()), stage_tpi(stages.size());
  std::vector<uint32_t> step_items(n_steps, 0);
  // a claim and its wait cost a few microseconds: small stages get a few tiles per item
  // (an NTT tile is a few microseconds of work, a leaf tile of 256 rows much more)
  for (size_t i = 0; i < stages.size(); i++) {
    const uint64_t tiles = tiles_of[i];
    const uint64_t min_tiles = stages[i].kind == LEAF ? 1 : stages[i].kind == COMP ? 2 : 4;
    const uint64_t tpi = std::min<uint64_t>(
        tiles, std::max<uint64_t>(min_tiles, (tiles + target_items - 1) / target_items));
    stage_tpi[i] = (uint32_t)tpi;
    stage_items[i] = (uint32_t)((tiles + tpi - 1) / tpi);
    step_items[stages[i].step] += stage_items[i];
  }
  for (auto &st : stages) st.dep_target = st.dep == NONE ? 0 : step_items[st.dep];
  // queue order: rounds ascending; within a round a wavefront over the traces' steps (step
  // k of every trace of the round, in the given order, then step k + 1)
  int max_round = 0;
  for (auto &tr : traces) max_round = std::max(max_round, tr.round);
  std::vector<Item> items;
  std::vector<uint32_t> first_item_of_stage(stages.size(), NONE), last_item_of_step(n_steps, 0);
  for (int r = 0; r <= max_round; r++) {
    size_t max_steps = 0;
    for (size_t t = 0; t < traces.size(); t++)
      if (traces[t].round == r) max_steps = std::max(max_steps, trace_steps[t].size());
    for (size_t k = 0; k < max_steps; k++)
      for (size_t t = 0; t < traces.size(); t++) {
        if (traces[t].round != r || k >= trace_steps[t].size()) continue;
        for (uint32_t si : step_stages[trace_steps[t][k]]) {
          const uint64_t tiles = tiles_of[si];
          first_item_of_stage[si] = (uint32_t)items.size();
          for (uint64_t a = 0; a < tiles; a += stage_tpi[si])
            items.push_back(Item{si, (uint32_t)a, (uint32_t)std::min<uint64_t>(stage_tpi[si], tiles - a)});
          last_item_of_step[stages[si].step] = (uint32_t)items.size() - 1;
        }
      }
  }
  ZKB_REQUIRE(items.size() < NONE - 1, "internal: %zu work items", items.size());
  // consistency of the queue before anything runs: every item inside its stage's tiles,
  // every counter index inside the table, every dependency on an earlier step of the
  // same trace (so on items earlier in the queue)
  {
    std::vector<uint64_t> covered(stages.size(), 0);
    for (const Item &it : items) {
      ZKB_REQUIRE(it.stage < stages.size() && it.ntiles >= 1 &&
                      (uint64_t)it.tile0 + it.ntiles <= tiles_of[it.stage],
                  "internal: work item outside its stage");
      covered[it.stage] += it.ntiles;
    }
    for (size_t i = 0; i < stages.size(); i++) {
      ZKB_REQUIRE(covered[i] == tiles_of[i], "internal: stage %zu tiles %llu, items cover %llu", i,
                  (unsigned long long)tiles_of[i], (unsigned long long)covered[i]);
      ZKB_REQUIRE(stages[i].step < n_steps && (stages[i].dep == NONE || stages[i].dep < stages[i].step),
                  "internal: stage %zu counters", i);
      // the dependency's items all come earlier in the queue than this stage's
      ZKB_REQUIRE(stages[i].dep == NONE || last_item_of_step[stages[i].dep] < first_item_of_stage[i],
                  "internal: stage %zu waits on a later item", i);
      ZKB_REQUIRE(stages[i].dep == NONE || stages[i].dep_target == step_items[stages[i].dep],
                  "internal: stage %zu dependency target", i);
    }
  }

  // ---- device tables: w_64 tables | stages | stalled copy | items | head, error, counters
  // (+1 never bumped)
  const size_t stw_off = 0;
  stages_off_ = align256(2 * sizeof(SmallTw<BabyBear>));
  stall_off_ = stages_off_ + align256(stages.size() * sizeof(Stage));
  items_off_ = stall_off_ + align256(stages.size() * sizeof(Stage));
  ctr_off_ = items_off_ + align256(items.size() * sizeof(Item));
  n_ctr_ = 2 + n_steps + 1;
  const size_t bytes = ctr_off_ + align256(n_ctr_ * sizeof(uint32_t));
  if (d_) {
    cudaFree(d_);
    d_ = nullptr;
  }
  note_device_alloc();
  ZKB_CHECK_CUDA(cudaMalloc(&d_, bytes));
  char *b = (char *)d_;
  SmallTw<BabyBear> stw[2];
  small_twiddles_bb(true, &stw[0]);
  small_twiddles_bb(false, &stw[1]);
  const SmallTw<BabyBear> *d_stw = (const SmallTw<BabyBear> *)(b + stw_off);
  for (auto &st : stages) {
    st.sti = d_stw;
    st.stf = d_stw + 1;
  }
  ZKB_CHECK_CUDA(cudaMemcpyAsync(b + stw_off, stw, sizeof stw, cudaMemcpyHostToDevice, s));
  // the stalled copy: the first stage with a dependency waits on the counter nothing bumps
  std::vector<Stage> stalled = stages;
  for (auto &st : stalled)
    if (st.dep != NONE) {
      st.dep = n_steps;  // counter index n_steps: never bumped
      st.dep_target = 1;
      break;
    }
  ZKB_CHECK_CUDA(cudaMemcpyAsync(b + stages_off_, stages.data(), stages.size() * sizeof(Stage),
                                 cudaMemcpyHostToDevice, s));
  ZKB_CHECK_CUDA(cudaMemcpyAsync(b + stall_off_, stalled.data(), stalled.size() * sizeof(Stage),
                                 cudaMemcpyHostToDevice, s));
  ZKB_CHECK_CUDA(cudaMemcpyAsync(b + items_off_, items.data(), items.size() * sizeof(Item),
                                 cudaMemcpyHostToDevice, s));
  ZKB_TRY(wait_stream(s));  // the host tables are staged; the NTT tables are built

  Params prm{};
  prm.stages = (const Stage *)(b + stages_off_);
  prm.items = (const Item *)(b + items_off_);
  prm.n_items = (uint32_t)items.size();
  prm.counters = (uint32_t *)(b + ctr_off_) + 2;
  prm.spin_limit = 0;
  prm.prof = nullptr;
  item_kind_.resize(items.size());
  for (size_t i = 0; i < items.size(); i++) item_kind_[i] = stages[items[i].stage].kind;
  if (d_prof_) {
    cudaFree(d_prof_);
    d_prof_ = nullptr;
  }
  prm.p2 = p2;
  host_params_.resize(sizeof(Params));
  memcpy(host_params_.data(), &prm, sizeof(Params));
  fusion_ = fusion;
  st_.stages = (uint32_t)stages.size();
  st_.steps = n_steps;
  st_.items = (uint32_t)items.size();
  st_.grid = (uint32_t)std::min<uint64_t>(resident, items.size());
  return ZKB_OK;
}

int PersistPlan::launch(cudaStream_t s, const void *stages, uint64_t spin_limit) const {
  ZKB_REQUIRE(d_ != nullptr, "persistent plan not built");
  Params prm;
  memcpy(&prm, host_params_.data(), sizeof(Params));
  prm.stages = (const Stage *)stages;
  prm.spin_limit = spin_limit;
  ZKB_CHECK_CUDA(cudaMemsetAsync((char *)d_ + ctr_off_, 0, n_ctr_ * sizeof(uint32_t), s));
  ZKB_LAUNCH("batch_persistent", s, persist_kernel<<<st_.grid, PT, smem_, s>>>(prm));
  return ZKB_OK;
}

int PersistPlan::enqueue(cudaStream_t s) const { return launch(s, (const char *)d_ + stages_off_, SPIN_LIMIT); }

int PersistPlan::enqueue_stalled(cudaStream_t s, uint64_t spin_limit) const {
  return launch(s, (const char *)d_ + stall_off_, spin_limit);
}

int PersistPlan::profile(cudaStream_t s, double ms_by_kind[4], double *span_ms) {
  ZKB_REQUIRE(d_ != nullptr, "persistent plan not built");
  const size_t bytes = (size_t)st_.items * 16;
  if (!d_prof_) {
    note_device_alloc();
    ZKB_CHECK_CUDA(cudaMalloc(&d_prof_, bytes));
  }
  Params prm;
  memcpy(&prm, host_params_.data(), sizeof(Params));
  prm.spin_limit = SPIN_LIMIT;
  prm.prof = (uint64_t *)d_prof_;
  ZKB_CHECK_CUDA(cudaMemsetAsync(d_prof_, 0, bytes, s));
  ZKB_CHECK_CUDA(cudaMemsetAsync((char *)d_ + ctr_off_, 0, n_ctr_ * sizeof(uint32_t), s));
  ZKB_LAUNCH("batch_persistent", s, persist_kernel<<<st_.grid, PT, smem_, s>>>(prm));
  std::vector<uint64_t> t((size_t)st_.items * 2);
  ZKB_CHECK_CUDA(cudaMemcpyAsync(t.data(), d_prof_, bytes, cudaMemcpyDeviceToHost, s));
  ZKB_TRY(check(s));
  uint64_t t0 = ~0ull, t1 = 0;
  for (int k = 0; k < 4; k++) ms_by_kind[k] = 0;
  for (size_t i = 0; i < st_.items; i++) {
    const uint64_t a = t[2 * i], b = t[2 * i + 1];
    if (!a || b < a) continue;
    t0 = std::min(t0, a);
    t1 = std::max(t1, b);
    ms_by_kind[item_kind_[i]] += (b - a) * 1e-6;
  }
  *span_ms = t1 > t0 ? (t1 - t0) * 1e-6 : 0;
  return ZKB_OK;
}

int PersistPlan::check(cudaStream_t s) const {
  ZKB_REQUIRE(d_ != nullptr, "persistent plan not built");
  uint32_t err = 0;
  ZKB_CHECK_CUDA(cudaMemcpyAsync(&err, (const char *)d_ + ctr_off_ + sizeof(uint32_t), sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, s));
  ZKB_TRY(wait_stream(s));
  if (err) {
    set_error("persistent batch kernel: work item %u waited longer than its spin limit; the run's results are "
              "invalid",
              err - 1);
    return ZKB_ERR_TIMEOUT;
  }
  return ZKB_OK;
}

}  // namespace zkb
