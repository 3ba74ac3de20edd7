// fri.cu — FRI folding by 2 (base field and the BabyBear quartic extension).
//
// Base field: FriAccelerator::fold_* / MetalFri (zkf-core/src/acceleration.rs:197-217,
// zkf-metal/src/shaders/fri.metal:14-53):
//   out[i] = (e[2i] + e[2i+1]) / 2 + alpha * (e[2i] - e[2i+1]) * inv_tw[i].
// Extension: p3 TwoAdicFriFolding::fold_matrix with arity 2 over
// BinomialExtensionField<BabyBear, 4> (x^4 = 11):
//   out[i] = (r0 + r1)/2 + (beta/2) * g^-rev(i) * (r0 - r1),  g = w_{2 n_out},
// the rows (r0, r1) being the values at +x and -x of the bit-reversed domain.
#include <array>
#include <memory>

#include "common.cuh"
#include "engine.cuh"
#include "multitree.cuh"
#include "field.cuh"

namespace zkb {

// canonical x canonical -> canonical
template <class F>
__device__ __forceinline__ typename F::T mul_cc(typename F::T a, typename F::T b);
template <>
__device__ __forceinline__ uint32_t mul_cc<BabyBear>(uint32_t a, uint32_t b) {
  return BabyBear::mont(BabyBear::mont(a, b), BabyBear::R2);
}
template <>
__device__ __forceinline__ uint64_t mul_cc<Goldilocks>(uint64_t a, uint64_t b) {
  return Goldilocks::mul(a, b);
}

// inv_tw given (canonical): the reference formula verbatim.
template <class F>
__global__ void fri_fold_given_kernel(const typename F::T *__restrict__ e, typename F::T *__restrict__ out,
                                      uint64_t n_out, typename F::T alpha_enc,
                                      typename F::T inv2_enc,
                                      const typename F::T *__restrict__ inv_tw) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x) {
    typename F::T a = e[2 * i], b = e[2 * i + 1];
    typename F::T sum = F::mul_tw(F::add(a, b), inv2_enc);
    typename F::T d = F::mul_tw(mul_cc<F>(F::sub(a, b), inv_tw[i]), alpha_enc);
    out[i] = F::add(sum, d);
  }
}

// inv_tw computed: inv_tw[i] = g^-rev(i) / 2 from the cached inverse table of size 2*n_out.
template <class F>
__global__ void fri_fold_p3_kernel(const typename F::T *__restrict__ e, typename F::T *__restrict__ out,
                                   uint64_t n_out, int log_n, typename F::T alpha_enc,
                                   typename F::T inv2_enc,
                                   const typename F::T *__restrict__ itw) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x) {
    typename F::T a = e[2 * i], b = e[2 * i + 1];
    uint64_t r = log_n ? (__brevll(i) >> (64 - log_n)) : 0;
    typename F::T d = F::mul_tw(F::mul_tw(F::sub(a, b), itw[r]), alpha_enc);
    out[i] = F::mul_tw(F::add(F::add(a, b), d), inv2_enc);
  }
}

template <class F>
int fri_fold_base_dev(const typename F::T *d_evals, size_t n_out, typename F::T alpha,
                      const typename F::T *d_inv_tw, typename F::T *d_out, cudaStream_t s) {
  using T = typename F::T;
  if (n_out == 0) return ZKB_OK;
  ZKB_REQUIRE(alpha < F::P, "alpha is not a canonical field element");
  const T inv2 = Dom<F>::encode(inv_host<F>(2));
  const T a_enc = Dom<F>::encode(alpha);
  if (d_inv_tw) {
    ZKB_LAUNCH("fri_fold", s, fri_fold_given_kernel<F><<<grid_for(n_out, 256), 256, 0, s>>>(d_evals, d_out, n_out, a_enc, inv2,
                                                                  d_inv_tw));
  } else {
    int log_n = ilog2_exact(n_out);
    ZKB_REQUIRE(log_n >= 0, "n_out must be a power of two when inv_twiddles is NULL");
    const T *itw;
    ZKB_TRY(get_twiddles<F>(log_n + 1, true, &itw, s));
    ZKB_LAUNCH("fri_fold", s, fri_fold_p3_kernel<F><<<grid_for(n_out, 256), 256, 0, s>>>(d_evals, d_out, n_out, log_n, a_enc,
                                                               inv2, itw));
  }
  ZKB_CHECK_LAUNCH();
  return ZKB_OK;
}

// ---------------------------------------------------------- quartic extension
struct Ext4 {
  uint32_t c[4];
};

// a * b with b encoded (Montgomery) coefficientwise; x^4 = 11.
__device__ __forceinline__ Ext4 ext4_mul_enc(const Ext4 &a, const Ext4 &b_enc) {
  using B = BabyBear;
  uint32_t p[7];
#pragma unroll
  for (int k = 0; k < 7; k++) p[k] = 0;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) p[i + j] = B::add(p[i + j], B::mont(a.c[i], b_enc.c[j]));
  Ext4 r;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const uint32_t h = p[k + 4];
    const uint32_t h2 = B::add(h, h), h4 = B::add(h2, h2), h8 = B::add(h4, h4);
    r.c[k] = B::add(p[k], B::add(B::add(h8, h2), h));  // + 11 h
  }
  r.c[3] = p[3];
  return r;
}

struct Ext4Params {
  Ext4 half_beta_enc;  // beta / 2, Montgomery-encoded coefficients
  uint32_t inv2_enc;
};

// Output i of the fold from the rows r0 = e[2i], r1 = e[2i+1] (n_out = 2^log_n outputs).
__device__ __forceinline__ uint4 fold_ext4_one(uint4 r0, uint4 r1, uint64_t i, int log_n, const Ext4Params &prm,
                                               const uint32_t *__restrict__ itw) {
  using B = BabyBear;
  uint64_t r = log_n ? (__brevll(i) >> (64 - log_n)) : 0;
  const uint32_t w = itw[r];
  Ext4 d;
  d.c[0] = B::mul_tw(B::sub(r0.x, r1.x), w);
  d.c[1] = B::mul_tw(B::sub(r0.y, r1.y), w);
  d.c[2] = B::mul_tw(B::sub(r0.z, r1.z), w);
  d.c[3] = B::mul_tw(B::sub(r0.w, r1.w), w);
  Ext4 t = ext4_mul_enc(d, prm.half_beta_enc);
  uint4 o;
  o.x = B::add(B::mul_tw(B::add(r0.x, r1.x), prm.inv2_enc), t.c[0]);
  o.y = B::add(B::mul_tw(B::add(r0.y, r1.y), prm.inv2_enc), t.c[1]);
  o.z = B::add(B::mul_tw(B::add(r0.z, r1.z), prm.inv2_enc), t.c[2]);
  o.w = B::add(B::mul_tw(B::add(r0.w, r1.w), prm.inv2_enc), t.c[3]);
  return o;
}

__global__ void fri_fold_ext4_kernel(const uint32_t *__restrict__ e, uint32_t *__restrict__ out,
                                     uint64_t n_out, int log_n, const Ext4Params prm,
                                     const uint32_t *__restrict__ itw) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 r0 = reinterpret_cast<const uint4 *>(e)[2 * i];
    const uint4 r1 = reinterpret_cast<const uint4 *>(e)[2 * i + 1];
    reinterpret_cast<uint4 *>(out)[i] = fold_ext4_one(r0, r1, i, log_n, prm, itw);
  }
}

// The next FRI layer's leaves while it is made.  Leaf j of a layer is the sponge digest
// of its codeword's rows 2j and 2j+1 flattened to 8 base elements (one permutation);
// with FOLD each thread first folds its four input rows 4j..4j+3 (the two pairs that
// become rows 2j and 2j+1) and stores them, so the new codeword is hashed from
// registers instead of being read back.  Without FOLD it hashes the codeword `e` itself
// (round 0).  n_leaves = 2^(log_out - 1), the output codeword holding 2^log_out rows.
template <bool FOLD>
__global__ void __launch_bounds__(128)
    fri_fold_hash_kernel(const uint32_t *__restrict__ e, uint32_t *__restrict__ out, uint64_t n_leaves, int log_out,
                         const Ext4Params prm, const uint32_t *__restrict__ itw, uint32_t *__restrict__ digests,
                         const __grid_constant__ P2Params<BabyBear, 16> p) {
  using D = Dom<BabyBear>;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_leaves;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 *in = reinterpret_cast<const uint4 *>(e);
    uint4 a, b;
    if constexpr (FOLD) {
      a = fold_ext4_one(in[4 * j], in[4 * j + 1], 2 * j, log_out, prm, itw);
      b = fold_ext4_one(in[4 * j + 2], in[4 * j + 3], 2 * j + 1, log_out, prm, itw);
      reinterpret_cast<uint4 *>(out)[2 * j] = a;
      reinterpret_cast<uint4 *>(out)[2 * j + 1] = b;
    } else {
      a = in[2 * j];
      b = in[2 * j + 1];
    }
    uint32_t st[16] = {D::enter(a.x), D::enter(a.y), D::enter(a.z), D::enter(a.w),
                       D::enter(b.x), D::enter(b.y), D::enter(b.z), D::enter(b.w), 0, 0, 0, 0, 0, 0, 0, 0};
    p2_permute<BabyBear, 16>(st, p);
    uint4 *dg = reinterpret_cast<uint4 *>(digests) + 2 * j;
    dg[0] = make_uint4(D::leave(st[0]), D::leave(st[1]), D::leave(st[2]), D::leave(st[3]));
    dg[1] = make_uint4(D::leave(st[4]), D::leave(st[5]), D::leave(st[6]), D::leave(st[7]));
  }
}

static int fold_params(const uint32_t beta[4], Ext4Params *prm) {
  const uint32_t inv2 = inv_host<BabyBear>(2);
  for (int k = 0; k < 4; k++) {
    ZKB_REQUIRE(beta[k] < BabyBear::P, "beta is not canonical");
    prm->half_beta_enc.c[k] = BabyBear::tw_encode(BabyBear::mul_host(beta[k], inv2));
  }
  prm->inv2_enc = BabyBear::tw_encode(inv2);
  return ZKB_OK;
}

// Leaves of the layer whose codeword (2^log_out rows) is cw_out: folded from cw_in with
// beta (stored into cw_out as well), or, with beta NULL, hashed from cw_in = cw_out.
static int fri_fold_hash_dev(const uint32_t *cw_in, uint32_t *cw_out, int log_out, const uint32_t *beta,
                             uint32_t *leaf_digests, const P2Params<BabyBear, 16> &p, cudaStream_t s) {
  const uint64_t n_leaves = 1ull << (log_out - 1);
  const unsigned grid = grid_for(n_leaves, 128, 1u << 30);  // one leaf per thread
  if (beta) {
    Ext4Params prm;
    ZKB_TRY(fold_params(beta, &prm));
    const uint32_t *itw;
    ZKB_TRY(get_twiddles<BabyBear>(log_out + 1, true, &itw, s));
    ZKB_LAUNCH("fri_fold_hash", s, fri_fold_hash_kernel<true><<<grid, 128, 0, s>>>(cw_in, cw_out, n_leaves, log_out, prm, itw, leaf_digests, p));
  } else {
    ZKB_LAUNCH("fri_leaf_hash", s, fri_fold_hash_kernel<false><<<grid, 128, 0, s>>>(cw_in, nullptr, n_leaves, log_out, Ext4Params{}, nullptr, leaf_digests, p));
  }
  return ZKB_OK;
}

int fri_fold_ext4_dev(const uint32_t *d_evals, size_t n_out, const uint32_t beta[4],
                      uint32_t *d_out, cudaStream_t s) {
  if (n_out == 0) return ZKB_OK;
  int log_n = ilog2_exact(n_out);
  ZKB_REQUIRE(log_n >= 0, "n_out must be a power of two");
  ZKB_REQUIRE(((uintptr_t)d_evals & 15) == 0 && ((uintptr_t)d_out & 15) == 0,
              "extension buffers must be 16-byte aligned");
  Ext4Params prm;
  ZKB_TRY(fold_params(beta, &prm));
  const uint32_t *itw;
  ZKB_TRY(get_twiddles<BabyBear>(log_n + 1, true, &itw, s));
  ZKB_LAUNCH("fri_fold_ext4", s, fri_fold_ext4_kernel<<<grid_for(n_out, 256), 256, 0, s>>>(d_evals, d_out, n_out, log_n, prm, itw));
  ZKB_CHECK_LAUNCH();
  return ZKB_OK;
}

template int fri_fold_base_dev<BabyBear>(const uint32_t *, size_t, uint32_t, const uint32_t *,
                                         uint32_t *, cudaStream_t);
template int fri_fold_base_dev<Goldilocks>(const uint64_t *, size_t, uint64_t, const uint64_t *,
                                           uint64_t *, cudaStream_t);

}  // namespace zkb

// ============================================================================
// FRI commit phase over the BabyBear quartic extension, with seeded challenges.
//
// Round r commits the current codeword (2^(log_n - r) extension elements in the
// bit-reversed domain order) as a matrix of 2^(log_n - r - 1) rows x 8 base
// elements — each row the pair (x, -x) flattened coefficient-wise, which is how
// ExtensionMmcs hands an extension matrix of width 2 to the base-field MMCS — then
// folds by 2 with beta_r (p3 commit_phase, minus the transcript: beta_r and the query
// indices come from SmallRng seeds).  Queries open, for each round, the row holding
// the pair of the queried index (index >> (r + 1)) and its sibling path, as p3's
// answer_query does with open_batch.
// ============================================================================
namespace zkb {

struct FriRoundDesc {
  const uint32_t *leaves;    // 2^(depth) rows x 8 u32
  const uint32_t *layers;    // digest layers of this round's tree (8 u32 per digest)
  uint64_t layer_off[40];    // in digests
  int depth;                 // log2(rows)
};

// One thread per (query, round): copies the opened row and the depth sibling digests.
__global__ void fri_gather_kernel(const FriRoundDesc *__restrict__ rounds, int n_rounds,
                                  const uint64_t *__restrict__ idx, int n_queries,
                                  uint32_t *__restrict__ rows_out, uint32_t *__restrict__ sib_out,
                                  const uint64_t *__restrict__ sib_off) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_queries * n_rounds) return;
  const int q = t / n_rounds, r = t % n_rounds;
  const FriRoundDesc &d = rounds[r];
  const uint64_t pair = (idx[q] >> r) >> 1;
  uint32_t *ro = rows_out + ((uint64_t)q * n_rounds + r) * 8;
#pragma unroll
  for (int k = 0; k < 8; k++) ro[k] = d.leaves[pair * 8 + k];
  uint32_t *so = sib_out + (uint64_t)q * sib_off[n_rounds] + sib_off[r];
  for (int l = 0; l < d.depth; l++) {
    const uint64_t j = (pair >> l) ^ 1ull;
    const uint32_t *dg = d.layers + (d.layer_off[l] + j) * 8;
#pragma unroll
    for (int k = 0; k < 8; k++) so[l * 8 + k] = dg[k];
  }
}

void FriProof::release_device() {
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  for (void *p : owned) dev_free(p, stream);
  owned.clear();
  cudaSetDevice(prev);
}

FriProof::~FriProof() { release_device(); }

int fri_commit_ext4_dev(const HasherSpec &spec, const uint32_t *d_codeword, int log_n, int log_final,
                        uint64_t challenge_seed, int num_queries, uint64_t query_seed,
                        FriProof *pf, cudaStream_t s, DuplexChallenger *ch) {
  ZKB_REQUIRE(spec.field == FIELD_BABYBEAR && spec.width == 16,
              "the extension FRI commits with the BabyBear width-16 hasher");
  ZKB_REQUIRE(log_final >= 0 && log_final < log_n && log_n <= 27,
              "need 0 <= log_final < log_n <= 27 (got %d, %d)", log_final, log_n);
  ZKB_REQUIRE(num_queries >= 0 && num_queries <= 4096, "num_queries out of range");
  ZKB_REQUIRE(((uintptr_t)d_codeword & 15) == 0, "codeword must be 16-byte aligned");
  P2Params<BabyBear, 16> p;
  const bool p_ok = build_p2_params<BabyBear, 16>(spec, &p);
  ZKB_REQUIRE(p_ok, "invalid Poseidon2 parameters");
  ZKB_CHECK_CUDA(cudaGetDevice(&pf->device));
  pf->stream = s;
  pf->log_n = log_n;
  pf->log_final = log_final;
  const int rounds = log_n - log_final;
  ZKB_REQUIRE(!ch || ch->spec.field == FIELD_BABYBEAR, "the transcript must be over BabyBear");
  // Seeded challenges: every beta is known up front, so the folds (each hashing the
  // leaves of the layer it makes) run back to back and the trees of all rounds are then
  // compressed together (one launch per tree level across the rounds, one root gather).
  // Transcript challenges: beta_r depends on round r's root, so the rounds run in order.
  pf->query_idx.resize(num_queries);
  if (!ch) {
    SmallRng rng(challenge_seed);
    for (int r = 0; r < rounds; r++) {
      std::array<uint32_t, 4> beta;
      for (auto &b : beta) b = sample_babybear(rng);
      pf->betas.push_back(beta);
    }
    SmallRng qr(query_seed);
    for (auto &q : pf->query_idx) q = qr.next_u64() >> (64 - log_n);
  }

  // ---- one device allocation: folded codewords, digest layers, roots, tables, query answers
  auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
  uint64_t off = 0;
  std::vector<uint64_t> cw_off(rounds + 1, 0), lay_off(rounds);
  for (int r = 1; r <= rounds; r++) {  // codeword of round r (round `rounds` is the final one)
    cw_off[r] = off;
    off = al(off + (16ull << (log_n - r)));
  }
  const uint64_t layers_base = off;
  uint64_t digests = 0;
  for (int r = 0; r < rounds; r++) {
    lay_off[r] = digests;
    digests += 2 * (1ull << (log_n - r - 1)) - 1;
  }
  off = al(off + digests * 32);
  const uint64_t roots_off = off;
  off = al(off + (uint64_t)rounds * 32);
  uint64_t n_comp = 0;
  for (int r = 0; r < rounds; r++) n_comp += (uint64_t)(log_n - r - 1);
  const uint64_t tables_off = off;
  off = al(off + rounds * sizeof(mt::LeafJob) + n_comp * sizeof(mt::CompJob) + rounds * 8ull);
  std::vector<uint64_t> sib_off(rounds + 1, 0);
  for (int r = 0; r < rounds; r++) sib_off[r + 1] = sib_off[r] + (uint64_t)(log_n - r - 1) * 8;
  pf->sib_per_query = sib_off[rounds];
  pf->query_rows.resize((size_t)num_queries * rounds * 8);
  pf->query_sibs.resize((size_t)num_queries * pf->sib_per_query);
  const uint64_t desc_off = off;
  off = al(off + rounds * sizeof(FriRoundDesc));
  const uint64_t idx_off = off;
  off = al(off + (uint64_t)num_queries * 8 + 8);
  const uint64_t soff_off = off;
  off = al(off + sib_off.size() * 8);
  const uint64_t rows_off = off;
  off = al(off + pf->query_rows.size() * 4 + 4);
  const uint64_t sibs_off = off;
  off = al(off + pf->query_sibs.size() * 4 + 4);
  void *arena = nullptr;
  ZKB_TRY(dev_alloc(&arena, off, s));
  pf->owned.push_back(arena);
  if (t_job_stages) t_job_stages->fri_alloc = std::chrono::steady_clock::now();
  char *base = (char *)arena;
  auto cw = [&](int r) -> const uint32_t * {
    return r == 0 ? d_codeword : (const uint32_t *)(base + cw_off[r]);
  };

  // ---- trees of every round: round r commits 2^(log_n-r-1) rows of 8 (sibling pairs)
  std::vector<const void *> data(rounds);
  std::vector<uint64_t> rows(rounds), widths(rounds, 8);
  std::vector<void *> layers(rounds);
  for (int r = 0; r < rounds; r++) {
    data[r] = cw(r);
    rows[r] = 1ull << (log_n - r - 1);
    layers[r] = base + layers_base + lay_off[r] * 32;
  }
  // Leaves: layer 0's are hashed from the input codeword; every later layer's leaves are
  // hashed by the kernel that folds the previous codeword into it (fri_fold_hash_dev),
  // so no codeword is read back to be hashed.  The last fold (into the final codeword)
  // has no layer after it.
  std::vector<std::vector<uint64_t>> layer_len(rounds);
  auto leaves = [&](int r) { return (uint32_t *)layers[r]; };
  ZKB_TRY(fri_fold_hash_dev(cw(0), nullptr, log_n, nullptr, leaves(0), p, s));
  if (!ch) {
    for (int r = 1; r < rounds; r++)
      ZKB_TRY(fri_fold_hash_dev(cw(r - 1), (uint32_t *)cw(r), log_n - r, pf->betas[r - 1].data(), leaves(r), p, s));
    ZKB_TRY(fri_fold_ext4_dev(cw(rounds - 1), 1ull << log_final, pf->betas[rounds - 1].data(),
                              (uint32_t *)cw(rounds), s));
    mt::Tables tab;
    mt::build_tables(data, rows, widths, layers, layers[0], 8, 4, &tab);
    mt::LeafJob *d_leaf;
    mt::CompJob *d_comp;
    uint64_t *d_root_off;
    ZKB_TRY(mt::upload_tables(tab, base + tables_off, s, &d_leaf, &d_comp, &d_root_off));
    ZKB_TRY((mt::launch_trees<BabyBear, 16>(tab, d_leaf, d_comp, d_root_off, layers[0], base + roots_off, p, 128,
                                            s, nullptr, "fri_compress", "fri_roots")));
    layer_len = tab.layer_len;
  } else {
    char *tslot = base + tables_off;
    uint32_t root[8];
    for (int r = 0; r < rounds; r++) {
      mt::Tables tab;
      mt::build_tables({data[r]}, {rows[r]}, {8}, {layers[r]}, layers[r], 8, 4, &tab);
      mt::LeafJob *d_leaf;
      mt::CompJob *d_comp;
      uint64_t *d_root_off;
      ZKB_TRY(mt::upload_tables(tab, tslot, s, &d_leaf, &d_comp, &d_root_off));
      tslot += tab.device_bytes();
      char *d_root = base + roots_off + (size_t)r * 32;
      ZKB_TRY((mt::launch_trees<BabyBear, 16>(tab, d_leaf, d_comp, d_root_off, layers[r], d_root, p, 128, s,
                                              nullptr, "fri_compress", "fri_roots")));
      ZKB_CHECK_CUDA(cudaMemcpyAsync(root, d_root, 32, cudaMemcpyDeviceToHost, s));
      ZKB_TRY(wait_stream(s));
      for (uint32_t v : root) ch->observe(v);
      std::array<uint32_t, 4> beta;
      for (auto &b : beta) b = (uint32_t)ch->sample();
      pf->betas.push_back(beta);
      if (r + 1 < rounds)
        ZKB_TRY(fri_fold_hash_dev(cw(r), (uint32_t *)cw(r + 1), log_n - r - 1, beta.data(), leaves(r + 1), p, s));
      else
        ZKB_TRY(fri_fold_ext4_dev(cw(r), 1ull << log_final, beta.data(), (uint32_t *)cw(r + 1), s));
      layer_len[r] = tab.layer_len[0];
    }
  }

  // ---- answers to the host: roots, final codeword, query openings
  if (t_job_stages) t_job_stages->fri_enqueued = std::chrono::steady_clock::now();
  pf->roots.resize((size_t)rounds * 8);
  ZKB_CHECK_CUDA(cudaMemcpyAsync(pf->roots.data(), base + roots_off, (size_t)rounds * 32, cudaMemcpyDeviceToHost, s));
  pf->final_cw.resize((1ull << log_final) * 4);
  ZKB_CHECK_CUDA(cudaMemcpyAsync(pf->final_cw.data(), cw(rounds), 16ull << log_final, cudaMemcpyDeviceToHost, s));
  if (ch) {
    // the final codeword goes into the transcript, then the query indices come out of it
    ZKB_TRY(wait_stream(s));
    for (uint32_t v : pf->final_cw) ch->observe(v);
    for (auto &q : pf->query_idx) q = ch->sample_bits(log_n);
  }
  if (num_queries > 0) {
    std::vector<FriRoundDesc> descs(rounds);
    for (int r = 0; r < rounds; r++) {
      FriRoundDesc &d = descs[r];
      d.leaves = cw(r);
      d.layers = (const uint32_t *)layers[r];
      d.depth = log_n - r - 1;
      ZKB_REQUIRE(d.depth < 40, "internal: FRI tree depth");
      uint64_t o = 0;
      for (int l = 0; l < d.depth; l++) {
        d.layer_off[l] = o;
        o += layer_len[r][l];
      }
    }
    ZKB_CHECK_CUDA(cudaMemcpyAsync(base + desc_off, descs.data(), descs.size() * sizeof(FriRoundDesc),
                                   cudaMemcpyHostToDevice, s));
    ZKB_CHECK_CUDA(cudaMemcpyAsync(base + idx_off, pf->query_idx.data(), num_queries * 8, cudaMemcpyHostToDevice, s));
    ZKB_CHECK_CUDA(cudaMemcpyAsync(base + soff_off, sib_off.data(), sib_off.size() * 8, cudaMemcpyHostToDevice, s));
    const int tasks = num_queries * rounds;
    ZKB_LAUNCH("fri_query_gather", s, fri_gather_kernel<<<(tasks + 127) / 128, 128, 0, s>>>((const FriRoundDesc *)(base + desc_off), rounds, (const uint64_t *)(base + idx_off), num_queries, (uint32_t *)(base + rows_off), (uint32_t *)(base + sibs_off), (const uint64_t *)(base + soff_off)));
    ZKB_CHECK_CUDA(cudaMemcpyAsync(pf->query_rows.data(), base + rows_off, pf->query_rows.size() * 4,
                                   cudaMemcpyDeviceToHost, s));
    ZKB_CHECK_CUDA(cudaMemcpyAsync(pf->query_sibs.data(), base + sibs_off, pf->query_sibs.size() * 4,
                                   cudaMemcpyDeviceToHost, s));
  }
  // the host tables above must outlive their (staged) uploads; the answers must be on the host
  ZKB_TRY(wait_stream(s));
  if (t_job_stages) t_job_stages->fri_answers = std::chrono::steady_clock::now();
  return ZKB_OK;
}

}  // namespace zkb

namespace zkb {

// out[i] = sum_j alpha^j * lde[i][j] over BabyBear^4.  One warp per row: lane l reads
// columns l, l+32, ... (coalesced; V4 = four consecutive columns per lane with 128-bit
// loads when the width is a multiple of 4), unrolled so that several loads are in
// flight per lane.  The powers arrive encoded as alpha^j * 2^64 mod p, so each
// Montgomery product is v * alpha^j * 2^32 and a lane's unreduced 64-bit sum of them
// (below p * 2^32 for any width < 2^29) needs one Montgomery reduction to come out as
// sum v * alpha^j; the 32 lane sums are then added mod p across the warp.
template <bool V4>
__global__ void __launch_bounds__(256)
    combine_columns_kernel(const uint32_t *__restrict__ lde, uint64_t rows, uint32_t width,
                           const uint4 *__restrict__ apow, uint4 *__restrict__ out) {
  using B = BabyBear;
  const unsigned lane = threadIdx.x & 31;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
    const uint32_t *row = lde + r * width;
    uint64_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    auto acc = [&](uint32_t v, uint4 w) {
      a0 += B::mont_lazy(v, w.x);
      a1 += B::mont_lazy(v, w.y);
      a2 += B::mont_lazy(v, w.z);
      a3 += B::mont_lazy(v, w.w);
    };
    // two columns per Montgomery reduction (v0 w0 + v1 w1 < 2p^2 < p 2^32)
    auto acc2 = [&](uint32_t v0, uint4 w0, uint32_t v1, uint4 w1) {
      a0 += B::mont_lazy_sum(v0, w0.x, v1, w1.x);
      a1 += B::mont_lazy_sum(v0, w0.y, v1, w1.y);
      a2 += B::mont_lazy_sum(v0, w0.z, v1, w1.z);
      a3 += B::mont_lazy_sum(v0, w0.w, v1, w1.w);
    };
    if constexpr (V4) {
#pragma unroll 2
      for (uint32_t j = 4 * lane; j < width; j += 128) {
        const uint4 v = *reinterpret_cast<const uint4 *>(row + j);
        acc2(v.x, apow[j], v.y, apow[j + 1]);
        acc2(v.z, apow[j + 2], v.w, apow[j + 3]);
      }
    } else {
#pragma unroll 4
      for (uint32_t j = lane; j < width; j += 32) acc(row[j], apow[j]);
    }
    uint32_t c0 = B::mont_reduce(a0), c1 = B::mont_reduce(a1), c2 = B::mont_reduce(a2),
             c3 = B::mont_reduce(a3);
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      c0 = B::add(c0, __shfl_xor_sync(0xffffffffu, c0, off));
      c1 = B::add(c1, __shfl_xor_sync(0xffffffffu, c1, off));
      c2 = B::add(c2, __shfl_xor_sync(0xffffffffu, c2, off));
      c3 = B::add(c3, __shfl_xor_sync(0xffffffffu, c3, off));
    }
    if (lane == 0) out[r] = make_uint4(c0, c1, c2, c3);
  }
}

static void ext4_mul_host(const uint32_t *a, const uint32_t *b, uint32_t *o) {
  uint64_t c[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) c[i + j] = (c[i + j] + (uint64_t)a[i] * b[j]) % BabyBear::P;
  for (int k = 0; k < 4; k++) o[k] = (uint32_t)((c[k] + 11 * (k + 4 < 7 ? c[k + 4] : 0)) % BabyBear::P);
}

int alpha_powers_dev(const uint32_t alpha[4], uint32_t width, ScratchBuf *out, cudaStream_t s) {
  for (int k = 0; k < 4; k++) ZKB_REQUIRE(alpha[k] < BabyBear::P, "alpha is not canonical");
  std::vector<uint32_t> pw((size_t)width * 4);
  uint32_t cur[4] = {1, 0, 0, 0};
  for (uint32_t j = 0; j < width; j++) {
    for (int k = 0; k < 4; k++) pw[j * 4 + k] = BabyBear::tw_encode(BabyBear::tw_encode(cur[k]));
    uint32_t nx[4];
    ext4_mul_host(cur, alpha, nx);
    for (int k = 0; k < 4; k++) cur[k] = nx[k];
  }
  ZKB_TRY(out->alloc(pw.size() * 4, s));
  ZKB_CHECK_CUDA(cudaMemcpyAsync(out->p, pw.data(), pw.size() * 4, cudaMemcpyHostToDevice, s));
  return ZKB_OK;  // a pageable source is staged before the copy call returns
}

int combine_columns_ext4_dev(const uint32_t *d_lde, uint64_t rows, uint32_t width,
                             const uint32_t alpha[4], uint32_t *d_out, cudaStream_t s) {
  ZKB_REQUIRE(((uintptr_t)d_out & 15) == 0, "output must be 16-byte aligned");
  ScratchBuf d_pw;
  ZKB_TRY(alpha_powers_dev(alpha, width, &d_pw, s));
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));
  ZKB_REQUIRE(width < (1u << 30), "width too large");
  const unsigned grid = grid_for(rows * 32, 256, (unsigned)ctx->sm_count * 8u);
  if (width % 4 == 0 && ((uintptr_t)d_lde & 15) == 0)
    ZKB_LAUNCH("combine_columns", s, combine_columns_kernel<true><<<grid, 256, 0, s>>>(d_lde, rows, width, d_pw.as<uint4>(), (uint4 *)d_out));
  else
    ZKB_LAUNCH("combine_columns", s, combine_columns_kernel<false><<<grid, 256, 0, s>>>(d_lde, rows, width, d_pw.as<uint4>(), (uint4 *)d_out));
  return ZKB_OK;
}

}  // namespace zkb
