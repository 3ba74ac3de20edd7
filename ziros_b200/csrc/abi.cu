// abi.cu — extern "C" entry points declared in include/zkb200.h.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

namespace zkb {
const char *last_error();
int measure_mul_peak(int field, double *mul_per_s);
}

using namespace zkb;



namespace {

// Declines (reference fallback semantics) when the process has no usable device.
int require_device() {
  ZKB_TRY(library_gate());
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error("no CUDA device available (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
    return ZKB_DECLINED;
  }
  return ZKB_OK;
}

#define ZKB_ENTRY() \
  clear_error();    \
  ZKB_TRY(require_device())

// Host buffer <-> device scratch helpers for the host-pointer entry points.
int to_device(ScratchBuf &buf, const void *host, size_t bytes, cudaStream_t s) {
  ZKB_TRY(buf.alloc(bytes, s));
  if (bytes) ZKB_CHECK_CUDA(cudaMemcpyAsync(buf.p, host, bytes, cudaMemcpyHostToDevice, s));
  return ZKB_OK;
}

int to_host(void *host, const void *dev, size_t bytes, cudaStream_t s) {
  if (bytes) ZKB_CHECK_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
  ZKB_TRY(wait_stream(s));
  return ZKB_OK;
}

template <class F>
int permute_dev_impl(typename F::T *d_states, size_t n_elems, const typename F::T *rc, size_t n_rc,
                     uint32_t n_ext, uint32_t n_int, cudaStream_t s) {
  ZKB_REQUIRE(n_elems % 16 == 0, "state buffer length %zu is not a multiple of 16", n_elems);
  ZKB_REQUIRE(rc != nullptr || n_rc == 0, "null round constants");
  const int field = sizeof(typename F::T) == 4 ? FIELD_BABYBEAR : FIELD_GOLDILOCKS;
  std::vector<uint64_t> rc64(rc, rc + n_rc);
  std::vector<uint64_t> diag = p2_diagonal(field, 16);
  P2Params<F, 16> p;
  if (!build_p2_params<F, 16>(rc64.data(), n_rc, (int)n_ext, (int)n_int, diag.data(), 8, &p)) {
    set_error("round constants do not match n_external_rounds=%u n_internal_rounds=%u (n_rc=%zu)",
              n_ext, n_int, n_rc);
    return ZKB_ERR_INVALID;
  }
  return p2_permute_batch<F, 16>(d_states, n_elems / 16, p, s);
}

template <class F>
int permute_host_impl(typename F::T *states, size_t n_elems, const typename F::T *rc, size_t n_rc,
                      uint32_t n_ext, uint32_t n_int) {
  using T = typename F::T;
  ZKB_REQUIRE(states != nullptr || n_elems == 0, "null states");
  cudaStream_t s = thread_stream();
  ScratchBuf d;
  ZKB_TRY(to_device(d, states, n_elems * sizeof(T), s));
  ZKB_TRY(permute_dev_impl<F>(d.as<T>(), n_elems, rc, n_rc, n_ext, n_int, s));
  return to_host(states, d.p, n_elems * sizeof(T), s);
}

int check_field(int field) {
  ZKB_REQUIRE(field == ZKB_FIELD_BABYBEAR || field == ZKB_FIELD_GOLDILOCKS, "unknown field %d", field);
  return ZKB_OK;
}

int hasher_spec(const zkb_hasher *h, HasherSpec *spec) {
  ZKB_REQUIRE(h != nullptr, "null hasher");
  ZKB_TRY(check_field(h->field));
  if (!make_hasher_spec(h->field, (int)h->width, h->seed, spec)) {
    set_error("unsupported Poseidon2 hasher: field %d width %u", h->field, h->width);
    return ZKB_ERR_UNSUPPORTED;
  }
  return ZKB_OK;
}

int tree_from(zkb_tree **tree_out, std::unique_ptr<zkb_tree> &tree, void *root_out, cudaStream_t s) {
  if (root_out) ZKB_TRY(mmcs_root_to_host(&tree->t, root_out, s));
  if (tree_out)
    *tree_out = tree.release();
  else
    ZKB_TRY(wait_stream(s));
  return ZKB_OK;
}

template <class F>
int fold_host(const typename F::T *evals, size_t n_evals, typename F::T alpha,
                     const typename F::T *inv_tw, typename F::T *out) {
  using T = typename F::T;
  ZKB_REQUIRE(n_evals % 2 == 0, "odd number of evaluations");
  ZKB_REQUIRE((evals && out) || n_evals == 0, "null buffers");
  const size_t n_out = n_evals / 2;
  cudaStream_t s = thread_stream();
  ScratchBuf de, dt, dout;
  ZKB_TRY(to_device(de, evals, n_evals * sizeof(T), s));
  if (inv_tw) ZKB_TRY(to_device(dt, inv_tw, n_out * sizeof(T), s));
  ZKB_TRY(dout.alloc(n_out * sizeof(T), s));
  ZKB_TRY(fri_fold_base_dev<F>(de.as<T>(), n_out, alpha, inv_tw ? dt.as<T>() : nullptr, dout.as<T>(), s));
  return to_host(out, dout.p, n_out * sizeof(T), s);
}

}  // namespace

extern "C" {

const char *zkb_version(void) { return "zkb200 0.1.0 (sm_100a)"; }

const char *zkb_last_error_message(void) { return last_error(); }

int zkb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int zkb_set_thresholds(const zkb_thresholds *t) {
  clear_error();
  set_thresholds(t ? *t : zkb_thresholds{});
  return ZKB_OK;
}

int zkb_get_thresholds(zkb_thresholds *t) {
  clear_error();
  ZKB_REQUIRE(t != nullptr, "null output");
  *t = thresholds();
  return ZKB_OK;
}

int zkb_circuit_open(char *why_out, size_t cap) {
  std::string why;
  const bool open = circuit_open(&why);
  if (why_out && cap) {
    std::snprintf(why_out, cap, "%s", open ? why.c_str() : "");
  }
  return open ? 1 : 0;
}

void zkb_circuit_reset(void) { circuit_reset(); }

int zkb_debug_inject_fault(int kind, int count) {
  clear_error();
  const int rc = inject_fault(kind, count);
  if (rc != ZKB_OK) set_error("unknown fault kind %d or negative count", kind);
  return rc;
}

uint64_t zkb_debug_device_allocations(void) { return device_alloc_count(); }
uint64_t zkb_debug_pool_allocations(void) { return pool_alloc_count(); }

int zkb_release_cached_memory(void) {
  clear_error();
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return ZKB_OK;
  return release_cached_memory();
}

int zkb_set_device(int device) {
  clear_error();
  ZKB_CHECK_CUDA(cudaSetDevice(device));
  return ZKB_OK;
}

int zkb_measure_mul_peak(int field, double *mul_per_s) {
  ZKB_ENTRY();
  ZKB_TRY(check_field(field));
  ZKB_REQUIRE(mul_per_s != nullptr, "null output");
  return measure_mul_peak(field, mul_per_s);
}

int zkb_profile_start(void) {
  clear_error();
  return profile_start();
}

int zkb_profile_stop(zkb_kernel_stat *out, int cap) {
  clear_error();
  ZKB_REQUIRE(out != nullptr || cap == 0, "null output");
  return profile_stop(out, cap);
}

// ------------------------------------------------------------------ Poseidon2
int zkb_poseidon2_babybear_round_constants(uint64_t seed, uint32_t *out, size_t cap,
                                           uint32_t *n_ext, uint32_t *n_int) {
  clear_error();
  int rf, rp;
  p2_round_numbers(FIELD_BABYBEAR, 16, &rf, &rp);
  std::vector<uint64_t> flat = p2_flat_constants(FIELD_BABYBEAR, 16, seed);
  ZKB_REQUIRE(out != nullptr && cap >= flat.size(), "output capacity %zu < %zu", cap, flat.size());
  for (size_t i = 0; i < flat.size(); i++) out[i] = (uint32_t)flat[i];
  if (n_ext) *n_ext = (uint32_t)rf;
  if (n_int) *n_int = (uint32_t)rp;
  return (int)flat.size();
}

int zkb_poseidon2_goldilocks_round_constants(uint64_t seed, uint32_t width, uint64_t *out,
                                             size_t cap, uint32_t *n_ext, uint32_t *n_int) {
  clear_error();
  int rf, rp;
  ZKB_REQUIRE(p2_round_numbers(FIELD_GOLDILOCKS, (int)width, &rf, &rp), "unsupported width %u", width);
  std::vector<uint64_t> flat = p2_flat_constants(FIELD_GOLDILOCKS, (int)width, seed);
  ZKB_REQUIRE(out != nullptr && cap >= flat.size(), "output capacity %zu < %zu", cap, flat.size());
  std::memcpy(out, flat.data(), flat.size() * 8);
  if (n_ext) *n_ext = (uint32_t)rf;
  if (n_int) *n_int = (uint32_t)rp;
  return (int)flat.size();
}

int zkb_poseidon2_babybear_permute(uint32_t *states, size_t n_elems, const uint32_t *rc, size_t n_rc,
                                   uint32_t n_ext, uint32_t n_int) {
  ZKB_ENTRY();
  ZKB_TRY(below(n_elems / 16, thresholds().poseidon2, "poseidon2"));
  return permute_host_impl<BabyBear>(states, n_elems, rc, n_rc, n_ext, n_int);
}

int zkb_poseidon2_goldilocks_permute(uint64_t *states, size_t n_elems, const uint64_t *rc,
                                     size_t n_rc, uint32_t n_ext, uint32_t n_int) {
  ZKB_ENTRY();
  ZKB_TRY(below(n_elems / 16, thresholds().poseidon2, "poseidon2"));
  return permute_host_impl<Goldilocks>(states, n_elems, rc, n_rc, n_ext, n_int);
}

int zkb_poseidon2_babybear_permute_dev(uint32_t *d_states, size_t n_elems, const uint32_t *rc,
                                       size_t n_rc, uint32_t n_ext, uint32_t n_int, void *stream) {
  ZKB_ENTRY();
  return permute_dev_impl<BabyBear>(d_states, n_elems, rc, n_rc, n_ext, n_int, resolve_stream(stream));
}

int zkb_poseidon2_goldilocks_permute_dev(uint64_t *d_states, size_t n_elems, const uint64_t *rc,
                                         size_t n_rc, uint32_t n_ext, uint32_t n_int,
                                         void *stream) {
  ZKB_ENTRY();
  return permute_dev_impl<Goldilocks>(d_states, n_elems, rc, n_rc, n_ext, n_int,
                                      resolve_stream(stream));
}

// ------------------------------------------------------------------------ DFT
int zkb_dft_batch_dev(int field, void *d, uint32_t log_h, uint32_t width, int inverse, void *stream) {
  ZKB_ENTRY();
  ZKB_TRY(check_field(field));
  cudaStream_t s = resolve_stream(stream);
  if (field == ZKB_FIELD_BABYBEAR)
    return ntt_dft_dev<BabyBear>((uint32_t *)d, (int)log_h, width, inverse != 0, s);
  return ntt_dft_dev<Goldilocks>((uint64_t *)d, (int)log_h, width, inverse != 0, s);
}

int zkb_set_ntt_tile_loads(int mode) {
  clear_error();
  ZKB_REQUIRE(mode == 0 || mode == 1, "tile load mode %d (0: loads into registers, 1: tensor copies)", mode);
  set_ntt_tile_loads(mode);
  return ZKB_OK;
}

int zkb_ntt_tile_load_errors(uint32_t *count) {
  ZKB_ENTRY();
  ZKB_REQUIRE(count != nullptr, "null count");
  return ntt_tma_wait_errors(count);
}

int zkb_dft_batch(int field, void *rowmajor, uint32_t log_h, uint32_t width, int inverse) {
  ZKB_ENTRY();
  ZKB_TRY(check_field(field));
  ZKB_REQUIRE(log_h < 40, "log_h too large");
  ZKB_TRY(below(1ull << log_h, thresholds().ntt, "ntt"));
  const size_t bytes = ((size_t)width << log_h) * field_elem_bytes(field);
  cudaStream_t s = thread_stream();
  ScratchBuf d;
  ZKB_TRY(to_device(d, rowmajor, bytes, s));
  ZKB_TRY(zkb_dft_batch_dev(field, d.p, log_h, width, inverse, s));
  return to_host(rowmajor, d.p, bytes, s);
}

int zkb_coset_lde_tuned_dev(int field, const void *d_trace, uint32_t log_h, uint32_t width,
                            uint32_t log_blowup, int kmax, uint32_t c_pass, uint32_t c_fused,
                            void *d_out, void *stream) {
  ZKB_ENTRY();
  ZKB_TRY(check_field(field));
  LdeTune t;
  t.kmax = kmax;
  t.c_pass = c_pass;
  t.c_fused = c_fused;
  ZKB_TRY(lde_tune_check(field, width, t));
  cudaStream_t s = resolve_stream(stream);
  if (field == ZKB_FIELD_BABYBEAR)
    return ntt_lde_dev<BabyBear>((const uint32_t *)d_trace, (int)log_h, width, (int)log_blowup,
                                 BabyBear::GENERATOR, true, (uint32_t *)d_out, s, &t);
  return ntt_lde_dev<Goldilocks>((const uint64_t *)d_trace, (int)log_h, width, (int)log_blowup,
                                 Goldilocks::GENERATOR, true, (uint64_t *)d_out, s, &t);
}

int zkb_coset_lde_batch_dev(int field, const void *d_trace, uint32_t log_h, uint32_t width,
                            uint32_t log_blowup, uint64_t shift, int bitrev_rows, void *d_out,
                            void *stream) {
  ZKB_ENTRY();
  ZKB_TRY(check_field(field));
  cudaStream_t s = resolve_stream(stream);
  if (field == ZKB_FIELD_BABYBEAR) {
    if (shift == 0) shift = BabyBear::GENERATOR;
    ZKB_REQUIRE(shift < BabyBear::P, "shift is not canonical");
    return ntt_lde_dev<BabyBear>((const uint32_t *)d_trace, (int)log_h, width, (int)log_blowup,
                                 (uint32_t)shift, bitrev_rows != 0, (uint32_t *)d_out, s);
  }
  if (shift == 0) shift = Goldilocks::GENERATOR;
  ZKB_REQUIRE(shift < Goldilocks::P, "shift is not canonical");
  return ntt_lde_dev<Goldilocks>((const uint64_t *)d_trace, (int)log_h, width, (int)log_blowup, shift,
                                 bitrev_rows != 0, (uint64_t *)d_out, s);
}

int zkb_coset_lde_batch(int field, const void *trace, uint32_t log_h, uint32_t width,
                        uint32_t log_blowup, uint64_t shift, int bitrev_rows, void *out) {
  ZKB_ENTRY();
  ZKB_TRY(check_field(field));
  ZKB_REQUIRE(log_h + log_blowup < 40, "size too large");
  ZKB_TRY(below(1ull << log_h, thresholds().ntt, "ntt"));
  const size_t es = field_elem_bytes(field);
  const size_t in_bytes = ((size_t)width << log_h) * es;
  const size_t out_bytes = in_bytes << log_blowup;
  cudaStream_t s = thread_stream();
  ScratchBuf din, dout;
  ZKB_TRY(to_device(din, trace, in_bytes, s));
  ZKB_TRY(dout.alloc(out_bytes, s));
  ZKB_TRY(zkb_coset_lde_batch_dev(field, din.p, log_h, width, log_blowup, shift, bitrev_rows, dout.p, s));
  return to_host(out, dout.p, out_bytes, s);
}

// ----------------------------------------------------------------------- MMCS
int zkb_mmcs_commit_dev(const zkb_hasher *hasher, const zkb_matrix *d_mats, size_t n_mats,
                        void *root_out, zkb_tree **tree_out, void *stream) {
  ZKB_ENTRY();
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(d_mats != nullptr && n_mats > 0, "No matrices given");
  cudaStream_t s = resolve_stream(stream);
  std::vector<TreeMatrix> mats;
  for (size_t i = 0; i < n_mats; i++) mats.push_back({d_mats[i].data, d_mats[i].height, d_mats[i].width});
  auto tree = std::make_unique<zkb_tree>();
  ZKB_TRY(mmcs_build_dev(spec, mats, &tree->t, s));
  return tree_from(tree_out, tree, root_out, s);
}

int zkb_mmcs_commit_reduce_dev(const zkb_hasher *hasher, const zkb_matrix *d_mat, const uint32_t *alpha,
                               void *root_out, zkb_tree **tree_out, uint32_t *d_codeword, void *stream) {
  ZKB_ENTRY();
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(spec.field == FIELD_BABYBEAR && spec.width == 16,
              "the fused alpha-reduction runs with the BabyBear width-16 hasher");
  ZKB_REQUIRE(d_mat != nullptr && d_mat->data != nullptr && d_mat->height > 0 && d_mat->width > 0 &&
                  alpha != nullptr && d_codeword != nullptr,
              "null or empty arguments");
  ZKB_REQUIRE(((uintptr_t)d_codeword & 15) == 0, "codeword must be 16-byte aligned");
  cudaStream_t s = resolve_stream(stream);
  std::vector<TreeMatrix> mats{{d_mat->data, d_mat->height, d_mat->width}};
  auto tree = std::make_unique<zkb_tree>();
  ScratchBuf apow;
  ZKB_TRY(alpha_powers_dev(alpha, (uint32_t)d_mat->width, &apow, s));
  const LeafCombine comb{apow.as<uint4>(), (uint4 *)d_codeword};
  ZKB_TRY(mmcs_build_dev(spec, mats, &tree->t, s, false, &comb));
  return tree_from(tree_out, tree, root_out, s);
}

int zkb_mmcs_commit(const zkb_hasher *hasher, const zkb_matrix *mats, size_t n_mats, void *root_out,
                    zkb_tree **tree_out) {
  ZKB_ENTRY();
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(mats != nullptr && n_mats > 0, "No matrices given");
  uint64_t leaves = 0;
  for (size_t i = 0; i < n_mats; i++) leaves = std::max<uint64_t>(leaves, mats[i].height);
  ZKB_TRY(below(leaves, thresholds().merkle, "merkle"));
  cudaStream_t s = thread_stream();
  auto tree = std::make_unique<zkb_tree>();
  tree->t.stream = s;
  ZKB_CHECK_CUDA(cudaGetDevice(&tree->t.device));
  const size_t es = field_elem_bytes(spec.field);
  std::vector<TreeMatrix> dm;
  for (size_t i = 0; i < n_mats; i++) {
    const size_t bytes = mats[i].height * mats[i].width * es;
    void *p = nullptr;
    ZKB_TRY(dev_alloc(&p, bytes ? bytes : 16, s));
    tree->t.owned.push_back(p);
    if (bytes) ZKB_CHECK_CUDA(cudaMemcpyAsync(p, mats[i].data, bytes, cudaMemcpyHostToDevice, s));
    dm.push_back({p, mats[i].height, mats[i].width});
  }
  ZKB_TRY(mmcs_build_dev(spec, dm, &tree->t, s));
  return tree_from(tree_out, tree, root_out, s);
}

namespace {
int pcs_commit_impl(const HasherSpec &spec, const void *d_trace, const void *h_trace, uint32_t log_h,
                    uint32_t width, uint32_t log_blowup, void *root_out, zkb_tree **tree_out,
                    cudaStream_t s, const uint32_t *alpha = nullptr, const zkb_fri_params *fri = nullptr,
                    FriProof *fri_out = nullptr, UploadGate *upload_mu = nullptr,
                    std::unique_lock<std::mutex> *compute_lock = nullptr, JobStages *stages = nullptr,
                    cudaStream_t fri_s = nullptr) {
  ZKB_REQUIRE(log_h + log_blowup < 40, "size too large");
  const size_t es = field_elem_bytes(spec.field);
  const uint64_t n = 1ull << log_h, N = n << log_blowup;
  auto tree = std::make_unique<zkb_tree>();
  tree->t.stream = s;
  ZKB_CHECK_CUDA(cudaGetDevice(&tree->t.device));
  // A host trace of at least two 64-column slabs (BabyBear, width-16 hasher) is uploaded a
  // slab at a time, and each slab's LDE and leaf absorption start once it has landed, while
  // the next slab crosses the link (see the leaf fill below).
  constexpr uint32_t kSlab = 64;
  const bool slabbed = h_trace && spec.field == FIELD_BABYBEAR && spec.width == 16 && width >= 2 * kSlab && log_h >= 1;
  ScratchBuf staged;
  if (h_trace) {
    ZKB_TRY(staged.alloc(n * width * es, s));
    if (slabbed) {
      // uploaded below, slab by slab
    } else if (upload_mu) {
      // one upload at a time: concurrent jobs would split the PCIe link and all start
      // computing late; serialised, each upload runs under the other jobs' kernels.  The
      // link is taken per 256 MiB piece, the upload with the fewest bytes left first, so a
      // small job's upload waits for one piece of a large job's, not for all of it.
      const size_t total = n * width * es, piece = 256ull << 20;
      const uint64_t ticket = upload_mu->ticket();
      for (size_t off = 0; off < total; off += piece) {
        const size_t len = total - off < piece ? total - off : piece;
        upload_mu->acquire(total - off, ticket);
        int rc = ZKB_OK;
        const cudaError_t e = cudaMemcpyAsync((char *)staged.p + off, (const char *)h_trace + off, len,
                                              cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
          set_error("cudaMemcpyAsync of a trace piece failed: %s", cudaGetErrorString(e));
          rc = ZKB_ERR_CUDA;
        }
        if (rc == ZKB_OK) rc = wait_stream(s);
        upload_mu->release();
        ZKB_TRY(rc);
      }
    } else {
      ZKB_CHECK_CUDA(cudaMemcpyAsync(staged.p, h_trace, n * width * es, cudaMemcpyHostToDevice, s));
    }
    d_trace = staged.p;
  }
  if (!slabbed) {
    if (stages) stages->uploaded = std::chrono::steady_clock::now();
    // an engine job waits here, its trace on the device, until the jobs of its size class
    // ahead of it have finished computing
    if (compute_lock) compute_lock->lock();
    if (stages) stages->lock_taken = std::chrono::steady_clock::now();
  }
  void *lde = nullptr;
  ZKB_TRY(dev_alloc(&lde, N * width * es, s));
  tree->t.owned.push_back(lde);
  // A staged copy of a host trace is ours: the inverse passes run in place on it
  // instead of in a separate coefficient scratch.
  int rc = ZKB_OK;
  if (slabbed)
    ;  // slab by slab in the leaf fill
  else if (spec.field == FIELD_BABYBEAR)
    rc = ntt_lde_dev<BabyBear>((const uint32_t *)d_trace, (int)log_h, width, (int)log_blowup,
                               BabyBear::GENERATOR, true, (uint32_t *)lde, s, nullptr,
                               h_trace ? staged.as<uint32_t>() : nullptr);
  else
    rc = ntt_lde_dev<Goldilocks>((const uint64_t *)d_trace, (int)log_h, width, (int)log_blowup,
                                 Goldilocks::GENERATOR, true, (uint64_t *)lde, s, nullptr,
                                 h_trace ? staged.as<uint64_t>() : nullptr);
  ZKB_TRY(rc);
  std::vector<TreeMatrix> mats{{lde, N, width}};
  // With seeded challenges alpha is known before the commitment, so the leaf hash does the
  // alpha-reduction while it reads each row (one pass over the LDE instead of two); with
  // the transcript alpha depends on the root and the reduction runs after the tree.
  void *cw = nullptr;
  const bool fused_reduction = fri && !fri->transcript && spec.field == FIELD_BABYBEAR && spec.width == 16;
  ScratchBuf apow;
  if (fri) {
    ZKB_REQUIRE(fri_out != nullptr, "internal: FRI job without a proof object");
    ZKB_TRY(dev_alloc(&cw, N * 16, s));
    fri_out->owned.push_back(cw);
    fri_out->stream = s;
    ZKB_CHECK_CUDA(cudaGetDevice(&fri_out->device));
  }
  if (fused_reduction) {
    ZKB_REQUIRE(alpha != nullptr, "null alpha");
    ZKB_TRY(alpha_powers_dev(alpha, width, &apow, s));
  }
  const LeafCombine comb{fused_reduction ? apow.as<uint4>() : nullptr, (uint4 *)cw};
  if (slabbed) {
    // Slab k (columns [64k, 64k + 64)) crosses the link on a copy stream of its own, in
    // pieces of at most 256 MiB through the engine's upload gate; once it has landed, its
    // LDE (inverse passes in place on the staged columns, row stride `width`) and the leaf
    // sponge over its columns (state carried between slabs, the alpha-reduction summed)
    // are enqueued on s, so they run while the next slab is copied.  An engine job takes
    // its size class's compute lock before its first slab's kernels if the lock is free,
    // else uploads every slab first and then waits for it, as an unslabbed job does.
    ScratchBuf carry;
    ZKB_TRY(carry.alloc(N * 16 * sizeof(uint32_t), s));
    struct StreamHolder {  // on an early return, no copy may still write into the staged trace
      cudaStream_t c = nullptr;
      ~StreamHolder() {
        if (c) {
          cudaStreamSynchronize(c);
          cudaStreamDestroy(c);
        }
      }
    } cs;
    ZKB_CHECK_CUDA(cudaStreamCreateWithFlags(&cs.c, cudaStreamNonBlocking));
    const uint32_t nslabs = (width + kSlab - 1) / kSlab;
    const LeafFill fill = [&](void *digests) -> int {
      uint32_t copied = 0, done = 0;
      bool locked = compute_lock == nullptr;
      auto compute = [&]() -> int {
        for (; done < copied; done++) {
          const uint32_t c0 = done * kSlab, nc = std::min(kSlab, width - c0);
          ZKB_TRY(ntt_lde_dev<BabyBear>(staged.as<uint32_t>() + c0, (int)log_h, nc, (int)log_blowup,
                                        BabyBear::GENERATOR, true, (uint32_t *)lde + c0, s, nullptr,
                                        staged.as<uint32_t>() + c0, width));
          ZKB_TRY(hash_rows_slab_dev(spec, (const uint32_t *)lde, width, c0, nc, N, carry.as<uint32_t>(), done == 0,
                                     done + 1 == nslabs, (uint32_t *)digests, fused_reduction ? &comb : nullptr, s));
        }
        return ZKB_OK;
      };
      const uint64_t total = n * width * es;
      uint64_t sent = 0;
      const uint64_t ticket = upload_mu ? upload_mu->ticket() : 0;
      for (uint32_t k = 0; k < nslabs; k++) {
        const uint32_t c0 = k * kSlab, nc = std::min(kSlab, width - c0);
        const uint64_t row_bytes = (uint64_t)nc * es;
        const uint64_t rows_per_piece = std::max<uint64_t>(1, (256ull << 20) / row_bytes);
        for (uint64_t r0 = 0; r0 < n; r0 += rows_per_piece) {
          const uint64_t rows = std::min<uint64_t>(rows_per_piece, n - r0);
          if (upload_mu) upload_mu->acquire(total - sent, ticket);
          const size_t off = (size_t)(r0 * width + c0) * es;
          int prc = ZKB_OK;
          const cudaError_t e = cudaMemcpy2DAsync((char *)staged.p + off, (size_t)width * es,
                                                  (const char *)h_trace + off, (size_t)width * es, row_bytes, rows,
                                                  cudaMemcpyHostToDevice, cs.c);
          if (e != cudaSuccess) {
            set_error("cudaMemcpy2DAsync of a trace slab failed: %s", cudaGetErrorString(e));
            prc = ZKB_ERR_CUDA;
          }
          if (prc == ZKB_OK) prc = wait_stream(cs.c);
          if (upload_mu) upload_mu->release();
          ZKB_TRY(prc);
          sent += rows * row_bytes;
        }
        copied++;
        if (!locked && compute_lock->try_lock()) {
          locked = true;
          if (stages) stages->lock_taken = std::chrono::steady_clock::now();
        }
        if (locked) ZKB_TRY(compute());
      }
      if (stages) stages->uploaded = std::chrono::steady_clock::now();
      if (!locked) {
        compute_lock->lock();
        if (stages) stages->lock_taken = std::chrono::steady_clock::now();
      }
      return compute();
    };
    ZKB_TRY(mmcs_build_dev(spec, mats, &tree->t, s, false, nullptr, &fill));
  } else if (fused_reduction) {
    ZKB_TRY(mmcs_build_dev(spec, mats, &tree->t, s, false, &comb));
  } else {
    ZKB_TRY(mmcs_build_dev(spec, mats, &tree->t, s));
  }
  if (compute_lock && compute_lock->owns_lock()) {
    // the large kernels (LDE, leaf hash, tree) are done when this returns; the FRI phase's
    // small kernels and host round trips overlap the next job's LDE
    ZKB_TRY(wait_stream(s));
    compute_lock->unlock();
  }
  if (stages) stages->tree_built = std::chrono::steady_clock::now();
  if (fri) {
    // alpha-reduction of the committed columns (unless fused above), then the FRI commit phase,
    // on fri_s when given: ordered after the tree by an event, and s waits for it before
    // anything of the job is read back or freed
    struct EventHolder {
      cudaEvent_t e = nullptr;
      ~EventHolder() {
        if (e) cudaEventDestroy(e);
      }
    } ev;
    cudaStream_t fs = s;
    if (fri_s && fri_s != s) {
      ZKB_CHECK_CUDA(cudaEventCreateWithFlags(&ev.e, cudaEventDisableTiming));
      ZKB_CHECK_CUDA(cudaEventRecord(ev.e, s));
      ZKB_CHECK_CUDA(cudaStreamWaitEvent(fri_s, ev.e, 0));
      fs = fri_s;
    }
    const int log_n = (int)(log_h + log_blowup);
    DuplexChallenger ch;
    uint32_t a[4];
    if (fri->transcript) {
      // the transcript sees the trace commitment before alpha is drawn
      uint32_t root[8];
      ZKB_TRY(mmcs_root_to_host(&tree->t, root, s));
      ZKB_TRY(ch.init(spec));
      for (uint32_t v : root) ch.observe(v);
      for (auto &x : a) x = (uint32_t)ch.sample();
    } else {
      ZKB_REQUIRE(alpha != nullptr, "null alpha");
      for (int k = 0; k < 4; k++) a[k] = alpha[k];
    }
    for (int k = 0; k < 4; k++) fri_out->alpha[k] = a[k];
    if (!fused_reduction) ZKB_TRY(combine_columns_ext4_dev((const uint32_t *)lde, N, width, a, (uint32_t *)cw, fs));
    ZKB_TRY(fri_commit_ext4_dev(spec, (const uint32_t *)cw, log_n, (int)fri->log_final,
                                fri->challenge_seed, (int)fri->num_queries, fri->query_seed, fri_out, fs,
                                fri->transcript ? &ch : nullptr));
    if (fs != s) {
      ZKB_CHECK_CUDA(cudaEventRecord(ev.e, fs));
      ZKB_CHECK_CUDA(cudaStreamWaitEvent(s, ev.e, 0));
    }
  }
  return tree_from(tree_out, tree, root_out, s);
}
}  // namespace

}  // extern "C"

thread_local zkb::JobStages *zkb::t_job_stages = nullptr;

// One engine job: host trace in, root (and the FRI answers) out, device state released
// before returning.
int zkb::pcs_job_run(const HasherSpec &spec, const void *h_trace, uint32_t log_h, uint32_t width,
                     uint32_t log_blowup, const uint32_t *alpha, const zkb_fri_params *fri, void *root_out,
                     FriProof *fri_out, cudaStream_t s, UploadGate *upload_mu, std::mutex *compute_mu,
                     JobStages *stages, cudaStream_t fri_stream) {
  t_job_stages = stages;
  std::unique_lock<std::mutex> cl;
  if (compute_mu) cl = std::unique_lock<std::mutex>(*compute_mu, std::defer_lock);
  int rc = pcs_commit_impl(spec, nullptr, h_trace, log_h, width, log_blowup, root_out, nullptr, s,
                           alpha, fri, fri_out, upload_mu, compute_mu ? &cl : nullptr, stages, fri_stream);
  if (fri_out) fri_out->release_device();
  if (rc == ZKB_OK) rc = wait_stream(s);
  if (stages) stages->released = std::chrono::steady_clock::now();
  t_job_stages = nullptr;
  return rc;  // the compute lock (if taken) is released here, after the job's work
}

extern "C" {

int zkb_pcs_commit(const zkb_hasher *hasher, const void *trace, uint32_t log_h, uint32_t width,
                   uint32_t log_blowup, void *root_out, zkb_tree **tree_out) {
  ZKB_ENTRY();
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(trace != nullptr && width > 0, "empty trace");
  ZKB_TRY(below(1ull << log_h, thresholds().ntt, "ntt"));
  return pcs_commit_impl(spec, nullptr, trace, log_h, width, log_blowup, root_out, tree_out,
                         thread_stream());
}

int zkb_pcs_commit_dev(const zkb_hasher *hasher, const void *d_trace, uint32_t log_h, uint32_t width,
                       uint32_t log_blowup, void *root_out, zkb_tree **tree_out, void *stream) {
  ZKB_ENTRY();
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(d_trace != nullptr && width > 0, "empty trace");
  return pcs_commit_impl(spec, d_trace, nullptr, log_h, width, log_blowup, root_out, tree_out,
                         resolve_stream(stream));
}

int zkb_pcs_commit_fri(const zkb_hasher *hasher, const void *trace, uint32_t log_h, uint32_t width,
                       uint32_t log_blowup, const uint32_t *alpha, const zkb_fri_params *params,
                       void *root_out, zkb_tree **tree_out, zkb_fri_proof **fri_out) {
  ZKB_ENTRY();
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(spec.field == FIELD_BABYBEAR, "the FRI job runs over the BabyBear quartic extension");
  ZKB_REQUIRE(trace != nullptr && width > 0 && alpha != nullptr && params != nullptr, "bad arguments");
  auto pf = std::make_unique<zkb_fri_proof>();
  ZKB_TRY(pcs_commit_impl(spec, nullptr, trace, log_h, width, log_blowup, root_out, tree_out,
                          thread_stream(), alpha, params, &pf->f));
  if (fri_out) *fri_out = pf.release();
  return ZKB_OK;
}

int zkb_pcs_commit_fri_dev(const zkb_hasher *hasher, const void *d_trace, uint32_t log_h, uint32_t width,
                           uint32_t log_blowup, const uint32_t *alpha, const zkb_fri_params *params,
                           void *root_out, zkb_tree **tree_out, zkb_fri_proof **fri_out, void *stream) {
  ZKB_ENTRY();
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(spec.field == FIELD_BABYBEAR, "the FRI job runs over the BabyBear quartic extension");
  ZKB_REQUIRE(d_trace != nullptr && width > 0 && alpha != nullptr && params != nullptr, "bad arguments");
  auto pf = std::make_unique<zkb_fri_proof>();
  ZKB_TRY(pcs_commit_impl(spec, d_trace, nullptr, log_h, width, log_blowup, root_out, tree_out,
                          resolve_stream(stream), alpha, params, &pf->f));
  if (fri_out) *fri_out = pf.release();
  return ZKB_OK;
}

const void *zkb_tree_matrix_dev(const zkb_tree *tree, int mat) {
  if (!tree || mat < 0 || mat >= (int)tree->t.mats.size()) return nullptr;
  return tree->t.mats[mat].data;
}

int zkb_tree_num_layers(const zkb_tree *tree) {
  if (!tree) return ZKB_ERR_INVALID;
  return (int)tree->t.layer_len.size();
}

int64_t zkb_tree_layer_len(const zkb_tree *tree, int layer) {
  if (!tree || layer < 0 || layer >= (int)tree->t.layer_len.size()) return ZKB_ERR_INVALID;
  return (int64_t)tree->t.layer_len[layer];
}

int zkb_tree_digest_elems(const zkb_tree *tree) {
  if (!tree) return ZKB_ERR_INVALID;
  return tree->t.spec.out;
}

int zkb_tree_copy_layer(const zkb_tree *tree, int layer, void *host_out) {
  clear_error();
  ZKB_REQUIRE(tree && layer >= 0 && layer < (int)tree->t.layer_len.size() && host_out,
              "invalid tree layer request");
  const DeviceTree &t = tree->t;
  const size_t es = field_elem_bytes(t.spec.field);
  const size_t D = t.spec.out;
  ZKB_CHECK_CUDA(cudaSetDevice(t.device));
  ZKB_CHECK_CUDA(cudaMemcpyAsync(host_out, (const char *)t.d_layers + t.layer_off[layer] * D * es,
                                 t.layer_len[layer] * D * es, cudaMemcpyDeviceToHost, t.stream));
  ZKB_TRY(wait_stream(t.stream));
  return ZKB_OK;
}

int zkb_mmcs_open_batch(const zkb_tree *tree, uint64_t index, void *rows_out, size_t rows_cap,
                        void *siblings_out, size_t siblings_cap) {
  clear_error();
  ZKB_REQUIRE(tree != nullptr, "null tree");
  const DeviceTree &t = tree->t;
  uint64_t max_h = 0, total_w = 0;
  for (const TreeMatrix &m : t.mats) {
    max_h = m.height > max_h ? m.height : max_h;
    total_w += m.width;
  }
  ZKB_REQUIRE(index < max_h, "index %llu out of bounds for height %llu", (unsigned long long)index,
              (unsigned long long)max_h);
  int log_max = 0;
  while ((1ull << log_max) < max_h) log_max++;
  const size_t es = field_elem_bytes(t.spec.field);
  const size_t D = t.spec.out;
  ZKB_REQUIRE(rows_out == nullptr || rows_cap >= total_w, "rows capacity %zu < %llu", rows_cap,
              (unsigned long long)total_w);
  ZKB_REQUIRE(siblings_out == nullptr || siblings_cap >= (size_t)log_max * D,
              "siblings capacity %zu < %zu", siblings_cap, (size_t)log_max * D);
  ZKB_CHECK_CUDA(cudaSetDevice(t.device));
  if (rows_out) {
    size_t off = 0;
    for (const TreeMatrix &m : t.mats) {
      int lh = 0;
      while ((1ull << lh) < m.height) lh++;
      const uint64_t r = index >> (log_max - lh);
      ZKB_CHECK_CUDA(cudaMemcpyAsync((char *)rows_out + off * es,
                                     (const char *)m.data + r * m.width * es, m.width * es,
                                     cudaMemcpyDeviceToHost, t.stream));
      off += m.width;
    }
  }
  if (siblings_out) {
    for (int i = 0; i < log_max; i++) {
      const uint64_t j = (index >> i) ^ 1ull;
      ZKB_REQUIRE(j < t.layer_len[i], "sibling outside layer %d", i);
      ZKB_CHECK_CUDA(cudaMemcpyAsync((char *)siblings_out + (size_t)i * D * es,
                                     (const char *)t.d_layers + (t.layer_off[i] + j) * D * es, D * es,
                                     cudaMemcpyDeviceToHost, t.stream));
    }
  }
  ZKB_TRY(wait_stream(t.stream));
  return ZKB_OK;
}

void zkb_tree_free(zkb_tree *tree) { delete tree; }

// ------------------------------------------------------------------------ FRI
int zkb_fri_fold_goldilocks(const uint64_t *evals, size_t n_evals, uint64_t alpha,
                            const uint64_t *inv_twiddles, uint64_t *out) {
  ZKB_ENTRY();
  ZKB_TRY(below(n_evals / 2, thresholds().fri, "fri"));
  return fold_host<Goldilocks>(evals, n_evals, alpha, inv_twiddles, out);
}

int zkb_fri_fold_babybear(const uint32_t *evals, size_t n_evals, uint32_t alpha,
                          const uint32_t *inv_twiddles, uint32_t *out) {
  ZKB_ENTRY();
  ZKB_TRY(below(n_evals / 2, thresholds().fri, "fri"));
  return fold_host<BabyBear>(evals, n_evals, alpha, inv_twiddles, out);
}

int zkb_fri_fold_babybear_ext4(const uint32_t *evals, size_t n_out, const uint32_t *beta, uint32_t *out) {
  ZKB_ENTRY();
  ZKB_REQUIRE(beta != nullptr && ((evals && out) || n_out == 0), "null buffers");
  cudaStream_t s = thread_stream();
  ScratchBuf de, dout;
  ZKB_TRY(to_device(de, evals, n_out * 8 * sizeof(uint32_t), s));
  ZKB_TRY(dout.alloc(n_out * 4 * sizeof(uint32_t), s));
  ZKB_TRY(fri_fold_ext4_dev(de.as<uint32_t>(), n_out, beta, dout.as<uint32_t>(), s));
  return to_host(out, dout.p, n_out * 4 * sizeof(uint32_t), s);
}

// ------------------------------------------------------------- FRI commit phase
namespace {
int fri_commit_impl(const zkb_hasher *hasher, const zkb_fri_params *prm, const uint32_t *d_cw,
                    zkb_fri_proof **out, cudaStream_t s) {
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(prm != nullptr && out != nullptr, "null arguments");
  auto pf = std::make_unique<zkb_fri_proof>();
  DuplexChallenger ch;
  if (prm->transcript) ZKB_TRY(ch.init(spec));
  ZKB_TRY(fri_commit_ext4_dev(spec, d_cw, (int)prm->log_n, (int)prm->log_final, prm->challenge_seed,
                              (int)prm->num_queries, prm->query_seed, &pf->f, s,
                              prm->transcript ? &ch : nullptr));
  *out = pf.release();
  return ZKB_OK;
}
}  // namespace

int zkb_fri_commit_babybear_ext4_dev(const zkb_hasher *hasher, const zkb_fri_params *params,
                                     const uint32_t *d_codeword, zkb_fri_proof **proof_out, void *stream) {
  ZKB_ENTRY();
  ZKB_REQUIRE(d_codeword != nullptr, "null codeword");
  return fri_commit_impl(hasher, params, d_codeword, proof_out, resolve_stream(stream));
}

int zkb_fri_commit_babybear_ext4_challenger_dev(const zkb_hasher *hasher, const zkb_fri_params *params,
                                                const uint32_t *d_codeword, zkb_challenger *challenger,
                                                zkb_fri_proof **proof_out, void *stream) {
  ZKB_ENTRY();
  ZKB_REQUIRE(d_codeword != nullptr && challenger != nullptr && params != nullptr && proof_out != nullptr,
              "null arguments");
  HasherSpec spec;
  ZKB_TRY(hasher_spec(hasher, &spec));
  ZKB_REQUIRE(spec.field == FIELD_BABYBEAR && challenger->c.spec.field == FIELD_BABYBEAR,
              "the FRI commit phase runs over BabyBear^4");
  auto pf = std::make_unique<zkb_fri_proof>();
  ZKB_TRY(fri_commit_ext4_dev(spec, d_codeword, (int)params->log_n, (int)params->log_final, 0,
                              (int)params->num_queries, 0, &pf->f, resolve_stream(stream), &challenger->c));
  *proof_out = pf.release();
  return ZKB_OK;
}

int zkb_fri_commit_babybear_ext4(const zkb_hasher *hasher, const zkb_fri_params *params,
                                 const uint32_t *codeword, zkb_fri_proof **proof_out) {
  ZKB_ENTRY();
  ZKB_REQUIRE(params != nullptr && codeword != nullptr && params->log_n < 31, "bad arguments");
  cudaStream_t s = thread_stream();
  ScratchBuf d;
  ZKB_TRY(to_device(d, codeword, (16ull << params->log_n), s));
  return fri_commit_impl(hasher, params, d.as<uint32_t>(), proof_out, s);
}

int zkb_fri_num_rounds(const zkb_fri_proof *p) {
  if (!p) return ZKB_ERR_INVALID;
  // counted from the host answers: the device trees may already have been released
  return (int)p->f.betas.size();
}

int zkb_fri_commitments(const zkb_fri_proof *p, uint32_t *roots_out, uint32_t *betas_out) {
  clear_error();
  ZKB_REQUIRE(p != nullptr, "null proof");
  if (roots_out) std::memcpy(roots_out, p->f.roots.data(), p->f.roots.size() * 4);
  if (betas_out)
    for (size_t r = 0; r < p->f.betas.size(); r++) std::memcpy(betas_out + 4 * r, p->f.betas[r].data(), 16);
  return ZKB_OK;
}

int zkb_fri_final_codeword(const zkb_fri_proof *p, uint32_t *out) {
  clear_error();
  ZKB_REQUIRE(p != nullptr && out != nullptr, "null arguments");
  std::memcpy(out, p->f.final_cw.data(), p->f.final_cw.size() * 4);
  return ZKB_OK;
}

int64_t zkb_fri_siblings_per_query(const zkb_fri_proof *p) {
  if (!p) return ZKB_ERR_INVALID;
  return (int64_t)p->f.sib_per_query;
}

int zkb_fri_query_openings(const zkb_fri_proof *p, uint64_t *indices_out, uint32_t *rows_out,
                           uint32_t *siblings_out) {
  clear_error();
  ZKB_REQUIRE(p != nullptr, "null proof");
  if (indices_out) std::memcpy(indices_out, p->f.query_idx.data(), p->f.query_idx.size() * 8);
  if (rows_out) std::memcpy(rows_out, p->f.query_rows.data(), p->f.query_rows.size() * 4);
  if (siblings_out) std::memcpy(siblings_out, p->f.query_sibs.data(), p->f.query_sibs.size() * 4);
  return ZKB_OK;
}

int zkb_fri_alpha(const zkb_fri_proof *p, uint32_t *alpha_out) {
  clear_error();
  ZKB_REQUIRE(p != nullptr && alpha_out != nullptr, "null arguments");
  std::memcpy(alpha_out, p->f.alpha.data(), 16);
  return ZKB_OK;
}

void zkb_fri_proof_free(zkb_fri_proof *p) { delete p; }

int zkb_combine_columns_babybear_ext4_dev(const uint32_t *d_lde, uint64_t rows, uint32_t width,
                                          const uint32_t *alpha, uint32_t *d_out, void *stream) {
  ZKB_ENTRY();
  ZKB_REQUIRE(d_lde != nullptr && d_out != nullptr && alpha != nullptr, "null arguments");
  return combine_columns_ext4_dev(d_lde, rows, width, alpha, d_out, resolve_stream(stream));
}

}  // extern "C"
