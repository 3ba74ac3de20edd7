// persist.cuh — the batched commitment as one persistent kernel fed by a device work queue.
#pragma once
#include <cstdint>
#include <vector>

#include "common.cuh"
#include "poseidon2.cuh"

namespace zkb {

// One BabyBear trace of a persistent plan: its device buffers (input, coefficient scratch,
// LDE, digest layers laid out layer after layer from the leaves, root) and shape.
struct PersistTrace {
  const uint32_t *in;
  uint32_t *coef;    // 2^log_h x width scratch of the inverse passes (unused with one pass),
                     // shared round-robin: `slot_prev` is the trace that used it before
  int slot_prev;     // index into the plan's traces, or -1; its LDE's fused step must have
                     // finished (the last read of the scratch) before this trace starts
  int round;         // queue order: rounds ascending, traces in the given order within one
  uint32_t *lde;     // 2^(log_h+log_b) x width, rows bit-reversed
  uint32_t *layers;  // 2 * rows - 1 digests of 8
  uint32_t *root;    // 8 elements
  int log_h;
  uint32_t width;    // multiple of 8
  int kmax;          // largest NTT pass (bits), at most 9
};

// Merkle-level fusion: levels computed by the tile that made the level below them, in
// shared memory.  leaf_levels: levels above the leaves done by the leaf-hash tile (0..8);
// comp_levels: levels per compression tile (1..8).
struct MerkleFusion {
  uint32_t leaf_levels = 0;
  uint32_t comp_levels = 1;
};

struct PersistStats {
  uint32_t stages = 0, steps = 0, items = 0, grid = 0;
};

class PersistPlan {
 public:
  PersistPlan() = default;
  PersistPlan(const PersistPlan &) = delete;
  PersistPlan &operator=(const PersistPlan &) = delete;
  ~PersistPlan();
  // Builds the stage and item tables (and every NTT table they read, on s; call outside a
  // capture) and uploads them.
  int build(const std::vector<PersistTrace> &traces, int log_b, const P2Params<BabyBear, 16> &p2,
            const MerkleFusion &fusion, cudaStream_t s);
  // Enqueues one run on s (capturable): clears the counters, launches the kernel.
  int enqueue(cudaStream_t s) const;
  // Host check after a run on s (waits for s): ZKB_ERR_TIMEOUT when a work item's wait gave up.
  int check(cudaStream_t s) const;
  // One run in which a work item waits on a counter that nothing bumps, with `spin_limit`
  // polls: exercises the bounded waits (the run's results are invalid; check() reports it).
  int enqueue_stalled(cudaStream_t s, uint64_t spin_limit) const;
  // One run (not captured) that records every item's start and end: the summed busy
  // time of the items by kind (NTT pass, fused LDE middle, leaf hash, compression), and the
  // span from the first start to the last end.
  int profile(cudaStream_t s, double ms_by_kind[4], double *span_ms);
  PersistStats stats() const { return st_; }
  MerkleFusion fusion() const { return fusion_; }

 private:
  int launch(cudaStream_t s, const void *stages, uint64_t spin_limit) const;
  void *d_ = nullptr;            // stages | stalled stages | items | counters, head, error
  size_t stages_off_ = 0, stall_off_ = 0, items_off_ = 0, ctr_off_ = 0, n_ctr_ = 0;
  size_t smem_ = 0;
  int device_ = 0;
  PersistStats st_;
  MerkleFusion fusion_;
  std::vector<unsigned char> host_params_;
  std::vector<uint8_t> item_kind_;
  void *d_prof_ = nullptr;
};

}  // namespace zkb
