// engine.cuh — internal host-side interfaces between the CUDA modules.
#pragma once
#include <chrono>
#include <map>
#include <array>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <set>
#include <vector>

#include "common.cuh"
#include "p2_consts.h"
#include "poseidon2.cuh"

namespace zkb {

// --------------------------------------------------------------- poseidon2.cu
template <class F, int W>
bool build_p2_params(const uint64_t *rc, size_t n_rc, int rounds_f, int rounds_p,
                     const uint64_t *diag, int out, P2Params<F, W> *p);
template <class F, int W>
bool build_p2_params(const HasherSpec &h, P2Params<F, W> *p);
template <class F, int W>
int p2_permute_batch(typename F::T *d_states, size_t n_states, const P2Params<F, W> &p,
                     cudaStream_t s);

// --------------------------------------------------------------------- ntt.cu
// Column-wise natural-order DFT of a row-major 2^log_h x width matrix, in place.
template <class F>
int ntt_dft_dev(typename F::T *d, int log_h, uint32_t width, bool inverse, cudaStream_t s);
// Kernel-shape choices of one LDE (zero = default): largest pass in index bits, columns
// per CTA of the plain passes and of the fused middle kernel.
struct LdeTune {
  int kmax = 0;
  uint32_t c_pass = 0;
  uint32_t c_fused = 0;
};
int lde_tune_check(int field, uint32_t width, const LdeTune &t);
// p3 coset_lde_batch (+ bit_reverse_rows when bitrev): d_out holds 2^(log_h+log_b) rows.
// coef_scratch (2^log_h x width), when given, is used instead of an allocation.  stride
// (0: width) is the row stride of d_trace, d_out and coef_scratch when the LDE covers
// `width` columns of wider matrices (bitrev only).
template <class F>
int ntt_lde_dev(const typename F::T *d_trace, int log_h, uint32_t width, int log_b,
                typename F::T shift, bool bitrev, typename F::T *d_out, cudaStream_t s,
                const LdeTune *tune = nullptr, typename F::T *coef_scratch = nullptr, uint32_t stride = 0);
// Natural-order DFT with caller-supplied twiddle (2^log_h) and temp (2^log_h x width) buffers.
template <class F>
int ntt_dft_into(typename F::T *d, int log_h, uint32_t width, bool inverse, typename F::T *tw_buf,
                 typename F::T *tmp, cudaStream_t s);
// Cached table of w^t (t < 2^log_n) for w = two_adic_generator(log_n)^(+-1), encoded
// for Field::mul_tw (Montgomery form for BabyBear).
template <class F>
int get_twiddles(int log_n, bool inverse, const typename F::T **out, cudaStream_t s);

// ------------------------------------------------------------------ merkle.cu
struct TreeMatrix {
  const void *data;  // device pointer, row-major
  uint64_t height;
  uint64_t width;
};

struct DeviceTree {
  HasherSpec spec;
  int device = 0;
  cudaStream_t stream = nullptr;
  void *d_layers = nullptr;                 // every digest layer, back to back
  std::vector<uint64_t> layer_off;          // in digests
  std::vector<uint64_t> layer_len;          // in digests
  std::vector<TreeMatrix> mats;             // commit order
  std::vector<void *> owned;                // device copies made by host-pointer commits
  bool borrowed = false;                    // d_layers lives in another object's arena
  ~DeviceTree();
};

// p3 MerkleTree::new over device matrices; fills layers and the tree description.
// fri_layer only renames the kernels for the timing hook (fri_leaf_hash / fri_compress).
// Alpha-reduction done by the leaf hash while it reads the rows (BabyBear width-16, one
// matrix): out[row] = sum_j alpha^j * row[j] in F_p^4, apow = alpha^j * 2^64 encoded
// (alpha_powers_dev).
struct LeafCombine {
  const uint4 *apow;
  uint4 *out;
};
// Writes a tree's layer 0 (the leaf digests) in place of the leaf-hash launch.
using LeafFill = std::function<int(void *digests)>;
int mmcs_build_dev(const HasherSpec &h, const std::vector<TreeMatrix> &mats, DeviceTree *tree,
                   cudaStream_t s, bool fri_layer = false, const LeafCombine *comb = nullptr,
                   const LeafFill *fill = nullptr);
// Leaf sponge over columns [c0, c0 + ncols) of a BabyBear matrix (width-16 hasher) arriving
// a slab at a time: state carried in `carry` (16 words per row) between slabs, digests on
// the last; with comb, the slab's alpha-reduction written (first) or added to comb->out.
int hash_rows_slab_dev(const HasherSpec &h, const uint32_t *mat, uint64_t stride, uint64_t c0, uint64_t ncols,
                       uint64_t height, uint32_t *carry, bool first, bool last, uint32_t *digests,
                       const LeafCombine *comb, cudaStream_t s);
// alpha^j * 2^64 mod p per coefficient, j < width, uploaded (uint4 per column).
int alpha_powers_dev(const uint32_t alpha[4], uint32_t width, ScratchBuf *out, cudaStream_t s);
// Copy the root (spec.out elements) to host memory (synchronises the stream).
int mmcs_root_to_host(const DeviceTree *tree, void *root_out, cudaStream_t s);

// --------------------------------------------------------------------- fri.cu
template <class F>
int fri_fold_base_dev(const typename F::T *d_evals, size_t n_out, typename F::T alpha,
                      const typename F::T *d_inv_tw, typename F::T *d_out, cudaStream_t s);
int fri_fold_ext4_dev(const uint32_t *d_evals, size_t n_out, const uint32_t beta[4],
                      uint32_t *d_out, cudaStream_t s);

// ---------------------------------------------------------------- challenger.cu
// Fiat-Shamir transcript: p3's DuplexChallenger<F, Poseidon2<16>, 16, 8> on the host.
struct DuplexChallenger {
  HasherSpec spec;
  P2Params<BabyBear, 16> p_bb;
  P2Params<Goldilocks, 16> p_gl;
  uint64_t state[16] = {0};
  std::vector<uint64_t> in, out;
  int init(const HasherSpec &s);
  void observe(uint64_t v);
  uint64_t sample();
  uint64_t sample_bits(int bits);

 private:
  void permute();
  void duplexing();
};

// FRI commit phase over BabyBear^4 and its query openings; the challenges are seeded
// draws, or come from a DuplexChallenger (transcript mode).
struct FriProof {
  int device = 0;
  cudaStream_t stream = nullptr;
  int log_n = 0, log_final = 0;
  std::vector<void *> owned;                       // device state: folded codewords, layer trees
  std::vector<std::array<uint32_t, 4>> betas;
  std::array<uint32_t, 4> alpha{};                 // alpha of the column reduction (commit+FRI jobs)
  std::vector<uint32_t> final_cw;                  // 2^log_final x 4, host
  std::vector<uint32_t> roots;                     // rounds x 8, host
  std::vector<uint64_t> query_idx;
  std::vector<uint32_t> query_rows;                // queries x rounds x 8
  std::vector<uint32_t> query_sibs;                // queries x sib_per_query
  uint64_t sib_per_query = 0;
  // Frees the device buffers (folded codewords, layer trees); host answers stay.
  void release_device();
  ~FriProof();
};

// Tile loads of the NTT passes (0 = coalesced loads into registers, 1 = one tensor copy
// per tile), and the count of tensor-copy waits that gave up (reset on read).
void set_ntt_tile_loads(int mode);
int ntt_tile_loads_mode();
int ntt_tma_wait_errors(uint32_t *count);

// The PCIe link of an engine, handed out one trace piece at a time.  Among the waiting
// uploads the one with the fewest bytes left goes next (ties: the earlier ticket, taken
// once per upload): an upload in progress keeps the link against a later one of equal size,
// so equal jobs upload one after another and the first starts computing early, while a
// small job's upload waits for at most one piece of a large one.  A waiting upload that
// pieces of later uploads have passed over `max_bypass` times goes next, so a steady stream
// of smaller uploads cannot hold a large job's upload (and the memory it was admitted with)
// back without bound; pieces of earlier uploads (the one in progress) do not count.
class UploadGate {
 public:
  explicit UploadGate(uint32_t max_bypass = 64) : max_bypass_(max_bypass) {}
  uint64_t ticket() {
    std::lock_guard<std::mutex> lk(mu_);
    return next_++;
  }
  void acquire(uint64_t bytes_left, uint64_t ticket) {
    std::unique_lock<std::mutex> lk(mu_);
    const std::pair<uint64_t, uint64_t> key{bytes_left, ticket};
    waiting_[key] = 0;
    cv_.wait(lk, [&] { return !busy_ && chosen() == key; });
    waiting_.erase(key);
    for (auto &w : waiting_)
      if (w.first.second < ticket) w.second++;  // an earlier upload was passed over
    busy_ = true;
  }
  void release() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      busy_ = false;
    }
    cv_.notify_all();
  }

 private:
  // the earliest upload passed over max_bypass times, else the fewest bytes left
  std::pair<uint64_t, uint64_t> chosen() const {
    const std::pair<uint64_t, uint64_t> *pick = nullptr;
    for (auto &w : waiting_)
      if (w.second >= max_bypass_ && (!pick || w.first.second < pick->second)) pick = &w.first;
    return pick ? *pick : waiting_.begin()->first;
  }
  std::mutex mu_;
  std::condition_variable cv_;
  std::map<std::pair<uint64_t, uint64_t>, uint32_t> waiting_;  // (bytes left, ticket) -> times passed over
  uint64_t next_ = 0;
  bool busy_ = false;
  const uint32_t max_bypass_;
};

// One PCS commit job from host memory (+ FRI when `fri` is set), device state released.
// upload_mu (may be NULL) serialises the host-to-device copies of concurrent jobs, taken
// per piece of the trace; compute_mu (may be NULL) is held from the end of the upload until
// the job's tree is built, so jobs sharing it run their large kernels one at a time while
// others upload (and their FRI phases overlap the next job's LDE).  fri_stream (may be NULL:
// s) runs the FRI phase; the engine gives it a higher priority than the next job's LDE and
// tree, whose long kernels would otherwise hold back its chain of small ones.
// Host times (steady clock) at which an engine job's stages ended, for the job log.
struct JobStages {
  std::chrono::steady_clock::time_point uploaded, lock_taken, tree_built;
  std::chrono::steady_clock::time_point fri_alloc, fri_enqueued, fri_answers, released;
};
// The stage record of the engine job running on this thread (null outside engine jobs).
extern thread_local JobStages *t_job_stages;
int pcs_job_run(const HasherSpec &spec, const void *h_trace, uint32_t log_h, uint32_t width,
                uint32_t log_blowup, const uint32_t *alpha, const zkb_fri_params *fri, void *root_out,
                FriProof *fri_out, cudaStream_t s, UploadGate *upload_mu = nullptr,
                std::mutex *compute_mu = nullptr, JobStages *stages = nullptr,
                cudaStream_t fri_stream = nullptr);
int combine_columns_ext4_dev(const uint32_t *d_lde, uint64_t rows, uint32_t width,
                             const uint32_t alpha[4], uint32_t *d_out, cudaStream_t s);
// With `ch` set, every round's root is observed before its beta is sampled, the final
// codeword is observed, and the query indices are sample_bits(log_n) (the seeds are
// then unused).
int fri_commit_ext4_dev(const HasherSpec &spec, const uint32_t *d_codeword, int log_n, int log_final,
                        uint64_t challenge_seed, int num_queries, uint64_t query_seed,
                        FriProof *pf, cudaStream_t s, DuplexChallenger *ch = nullptr);

}  // namespace zkb

// Opaque handles of the C ABI.
struct zkb_tree {
  zkb::DeviceTree t;
};

struct zkb_fri_proof {
  zkb::FriProof f;
};

struct zkb_challenger {
  zkb::DuplexChallenger c;
};
