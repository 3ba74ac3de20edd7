// verify.cu — Mmcs::verify_batch on the host.
//
// Checks one opening of a Poseidon2 MMCS commitment, exactly as the vendored p3
// MerkleTreeMmcs verifies it (vendor/p3-merkle-tree-gpu/src/mmcs.rs:230-330):
//   matrices sorted tallest first (stable); heights that round up to the same power of
//   two must be equal; the proof holds log2(next_pow2(max height)) siblings; the rows of
//   the tallest matrices are hashed together (PaddingFreeSponge over their concatenation),
//   then each sibling is compressed in on the side given by the index bit, and after each
//   level the rows of the matrices whose padded height matches the new level are hashed
//   and compressed in (injection); the result must equal the root.
// Verification is sequential and tiny (one sponge per height class, one compression per
// level), so it runs on the host with the permutation code the kernels use.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

namespace zkb {
namespace {

template <class F, int W>
struct HostHasher {
  using T = typename F::T;
  static constexpr int OUT = W == 16 ? 8 : 4;
  P2Params<F, W> p;

  // PaddingFreeSponge<Perm, W, 8, OUT> over a stream of canonical elements
  void sponge(const std::vector<T> &in, T *digest) const {
    T s[W];
    for (int i = 0; i < W; i++) s[i] = 0;
    for (size_t c = 0; c < in.size(); c += 8) {
      for (size_t i = 0; i < 8 && c + i < in.size(); i++) s[i] = Dom<F>::enter(in[c + i]);
      p2_permute<F, W>(s, p);
    }
    for (int i = 0; i < OUT; i++) digest[i] = Dom<F>::leave(s[i]);
  }
  // TruncatedPermutation<Perm, 2, OUT, W>
  void compress(const T *l, const T *r, T *out) const {
    T s[W];
    for (int i = 0; i < W; i++) s[i] = 0;
    for (int i = 0; i < OUT; i++) {
      s[i] = Dom<F>::enter(l[i]);
      s[OUT + i] = Dom<F>::enter(r[i]);
    }
    p2_permute<F, W>(s, p);
    for (int i = 0; i < OUT; i++) out[i] = Dom<F>::leave(s[i]);
  }
};

uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

template <class F, int W>
int verify_impl(const HasherSpec &spec, const void *root_v, const uint64_t *heights, const uint64_t *widths,
                size_t n, uint64_t index, const void *rows_v, const void *sibs_v, size_t n_sibs) {
  using T = typename F::T;
  constexpr int OUT = HostHasher<F, W>::OUT;
  HostHasher<F, W> h;
  ZKB_REQUIRE((build_p2_params<F, W>(spec, &h.p)), "invalid Poseidon2 parameters");
  const T *root = (const T *)root_v, *rows = (const T *)rows_v, *sibs = (const T *)sibs_v;
  // opened rows of matrix i start at offset[i] (commit order)
  std::vector<uint64_t> offset(n + 1, 0);
  for (size_t i = 0; i < n; i++) offset[i + 1] = offset[i] + widths[i];
  for (uint64_t k = 0; k < offset[n]; k++) ZKB_REQUIRE(rows[k] < F::P, "opened value %llu is not canonical",
                                                       (unsigned long long)k);
  std::vector<size_t> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return heights[a] > heights[b]; });
  for (size_t i = 0; i + 1 < n; i++) {
    const uint64_t a = heights[ord[i]], b = heights[ord[i + 1]];
    ZKB_REQUIRE(a == b || next_pow2(a) != next_pow2(b), "incompatible heights");
  }
  const uint64_t max_h = heights[ord[0]];
  uint64_t padded = next_pow2(max_h);
  int log_max = 0;
  while ((1ull << log_max) < padded) log_max++;
  ZKB_REQUIRE(n_sibs == (size_t)log_max, "wrong height: %zu siblings for log max height %d", n_sibs, log_max);
  ZKB_REQUIRE(index < max_h, "index %llu out of bounds for height %llu", (unsigned long long)index,
              (unsigned long long)max_h);
  size_t next = 0;
  auto take_rows = [&](auto pred) {
    std::vector<T> cat;
    while (next < n && pred(heights[ord[next]])) {
      const size_t m = ord[next++];
      cat.insert(cat.end(), rows + offset[m], rows + offset[m + 1]);
    }
    return cat;
  };
  T cur[OUT];
  h.sponge(take_rows([&](uint64_t ht) { return next_pow2(ht) == padded; }), cur);
  for (size_t l = 0; l < n_sibs; l++) {
    const T *sib = sibs + l * OUT;
    T nxt[OUT];
    if ((index & 1) == 0)
      h.compress(cur, sib, nxt);
    else
      h.compress(sib, cur, nxt);
    std::memcpy(cur, nxt, sizeof cur);
    index >>= 1;
    padded >>= 1;
    if (next < n && next_pow2(heights[ord[next]]) == padded) {
      const uint64_t ht = heights[ord[next]];
      T inj[OUT];
      h.sponge(take_rows([&](uint64_t x) { return x == ht; }), inj);
      h.compress(cur, inj, nxt);
      std::memcpy(cur, nxt, sizeof cur);
    }
  }
  for (int i = 0; i < OUT; i++)
    if (cur[i] != root[i]) {
      set_error("root mismatch");
      return ZKB_ERR_INVALID;
    }
  return ZKB_OK;
}

template <class F, int W>
int compress_impl(const HasherSpec &spec, const void *left, const void *right, size_t n, void *out) {
  using T = typename F::T;
  constexpr int OUT = HostHasher<F, W>::OUT;
  HostHasher<F, W> h;
  ZKB_REQUIRE((build_p2_params<F, W>(spec, &h.p)), "invalid Poseidon2 parameters");
  const T *l = (const T *)left, *r = (const T *)right;
  for (size_t k = 0; k < n * OUT; k++)
    ZKB_REQUIRE(l[k] < F::P && r[k] < F::P, "digest element %zu is not canonical", k);
  for (size_t i = 0; i < n; i++) h.compress(l + i * OUT, r + i * OUT, (T *)out + i * OUT);
  return ZKB_OK;
}

}  // namespace
}  // namespace zkb

using namespace zkb;

extern "C" int zkb_mmcs_compress(const zkb_hasher *hasher, const void *left, const void *right, size_t n,
                                 void *out) {
  clear_error();
  ZKB_REQUIRE(hasher && ((left && right && out) || n == 0), "null arguments");
  HasherSpec spec;
  if (!make_hasher_spec(hasher->field, (int)hasher->width, hasher->seed, &spec)) {
    set_error("unsupported Poseidon2 hasher: field %d width %u", hasher->field, hasher->width);
    return ZKB_ERR_UNSUPPORTED;
  }
  if (n == 0) return ZKB_OK;
  if (spec.field == FIELD_BABYBEAR) return compress_impl<BabyBear, 16>(spec, left, right, n, out);
  if (spec.width == 16) return compress_impl<Goldilocks, 16>(spec, left, right, n, out);
  return compress_impl<Goldilocks, 12>(spec, left, right, n, out);
}

extern "C" int zkb_mmcs_verify_batch(const zkb_hasher *hasher, const void *root, const uint64_t *heights,
                                     const uint64_t *widths, size_t n_mats, uint64_t index, const void *rows,
                                     const void *siblings, size_t n_siblings) {
  clear_error();
  ZKB_REQUIRE(hasher && root && heights && widths && n_mats > 0 && rows && (siblings || n_siblings == 0),
              "null arguments or empty batch");
  for (size_t i = 0; i < n_mats; i++) ZKB_REQUIRE(heights[i] > 0, "matrix height 0 not supported");
  HasherSpec spec;
  if (!make_hasher_spec(hasher->field, (int)hasher->width, hasher->seed, &spec)) {
    set_error("unsupported Poseidon2 hasher: field %d width %u", hasher->field, hasher->width);
    return ZKB_ERR_UNSUPPORTED;
  }
  if (spec.field == FIELD_BABYBEAR)
    return verify_impl<BabyBear, 16>(spec, root, heights, widths, n_mats, index, rows, siblings, n_siblings);
  if (spec.width == 16)
    return verify_impl<Goldilocks, 16>(spec, root, heights, widths, n_mats, index, rows, siblings, n_siblings);
  return verify_impl<Goldilocks, 12>(spec, root, heights, widths, n_mats, index, rows, siblings, n_siblings);
}
