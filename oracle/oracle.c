/*
 * oracle.c — CPU restatement of the ZirOS / Plonky3 0.4.2 polynomial-commitment
 * path (coset LDE, Poseidon2 Merkle commitment, FRI folding).
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA product.  It is
 * loaded by tests/, by __graft_entry__.smoke() and by the CPU-baseline legs of
 * bench.py, never by the product library.
 *
 * It restates the reference's CPU semantics in plain C, deliberately simple
 * (u64 / u128 remainder arithmetic, scalar loops, OpenMP across independent
 * columns and rows) so that it is easy to audit against the cited sources.
 * All paths are relative to the ZirOS repository root.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ========================================================================== */
/* Fields                                                                      */
/* BabyBear p = 2^31 - 2^27 + 1   (zkf-metal/src/shaders/field_babybear.metal:1-25) */
/* Goldilocks p = 2^64 - 2^32 + 1 (zkf-metal/src/shaders/field_goldilocks.metal:1-56) */
/* ========================================================================== */

uint32_t or_bb_add(uint32_t a, uint32_t b) {
  uint32_t s = a + b;
  return s >= OR_BB_P ? s - OR_BB_P : s;
}
uint32_t or_bb_sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + OR_BB_P - b; }
uint32_t or_bb_mul(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) % OR_BB_P); }
uint32_t or_bb_pow(uint32_t a, uint64_t e) {
  uint32_t r = 1, b = a;
  while (e) {
    if (e & 1) r = or_bb_mul(r, b);
    b = or_bb_mul(b, b);
    e >>= 1;
  }
  return r;
}
uint32_t or_bb_inv(uint32_t a) { return or_bb_pow(a, OR_BB_P - 2); }

uint64_t or_gl_add(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a + b) % OR_GL_P); }
uint64_t or_gl_sub(uint64_t a, uint64_t b) { return a >= b ? a - b : (uint64_t)((u128)a + OR_GL_P - b); }
uint64_t or_gl_mul(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % OR_GL_P); }
uint64_t or_gl_pow(uint64_t a, uint64_t e) {
  uint64_t r = 1, b = a;
  while (e) {
    if (e & 1) r = or_gl_mul(r, b);
    b = or_gl_mul(b, b);
    e >>= 1;
  }
  return r;
}
uint64_t or_gl_inv(uint64_t a) { return or_gl_pow(a, OR_GL_P - 2); }

/* Generic element ops over u64 carriers. */
static inline uint64_t f_add(int f, uint64_t a, uint64_t b) {
  return f == OR_FIELD_BABYBEAR ? or_bb_add((uint32_t)a, (uint32_t)b) : or_gl_add(a, b);
}
static inline uint64_t f_sub(int f, uint64_t a, uint64_t b) {
  return f == OR_FIELD_BABYBEAR ? or_bb_sub((uint32_t)a, (uint32_t)b) : or_gl_sub(a, b);
}
static inline uint64_t f_mul(int f, uint64_t a, uint64_t b) {
  return f == OR_FIELD_BABYBEAR ? or_bb_mul((uint32_t)a, (uint32_t)b) : or_gl_mul(a, b);
}
static inline uint64_t f_pow(int f, uint64_t a, uint64_t e) {
  return f == OR_FIELD_BABYBEAR ? or_bb_pow((uint32_t)a, e) : or_gl_pow(a, e);
}
static inline uint64_t f_inv(int f, uint64_t a) {
  return f == OR_FIELD_BABYBEAR ? or_bb_inv((uint32_t)a) : or_gl_inv(a);
}
static inline uint64_t f_modulus(int f) { return f == OR_FIELD_BABYBEAR ? OR_BB_P : OR_GL_P; }
static inline size_t f_esize(int f) { return f == OR_FIELD_BABYBEAR ? 4 : 8; }
static inline uint64_t ld(int f, const void *p, size_t i) {
  return f == OR_FIELD_BABYBEAR ? ((const uint32_t *)p)[i] : ((const uint64_t *)p)[i];
}
static inline void st(int f, void *p, size_t i, uint64_t v) {
  if (f == OR_FIELD_BABYBEAR)
    ((uint32_t *)p)[i] = (uint32_t)v;
  else
    ((uint64_t *)p)[i] = v;
}

/* Multiplicative generator: Goldilocks 7 (zkf-backends/src/wrapping/stark_to_groth16.rs:2333),
 * BabyBear 31 (p3-baby-bear GENERATOR; parity unpinned in-repo). */
uint64_t or_field_generator(int field) { return field == OR_FIELD_BABYBEAR ? 31 : 7; }

/* two_adic_generator(bits) = (g^((p-1)/2^S))^(2^(S-bits)) with S the two-adicity
 * (Goldilocks S = 32: stark_to_groth16.rs:2313-2322; BabyBear S = 27 by the same rule). */
uint64_t or_two_adic_generator(int field, int bits) {
  int S = field == OR_FIELD_BABYBEAR ? 27 : 32;
  uint64_t p = f_modulus(field);
  uint64_t root = f_pow(field, or_field_generator(field), (p - 1) >> S);
  for (int i = bits; i < S; i++) root = f_mul(field, root, root);
  return root;
}

/* ========================================================================== */
/* rand 0.9 SmallRng on 64-bit targets = Xoshiro256++ (Blackman & Vigna 2018);  */
/* seed_from_u64 expands the seed with SplitMix64 (Steele, Lea & Flood 2014).   */
/* Pinned through the Goldilocks golden vector                                  */
/* (zkf-backends/src/wrapping/poseidon2_goldilocks.rs:538-620).                 */
/* ========================================================================== */

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

void or_rng_seed(or_rng *r, uint64_t seed) {
  uint64_t state = seed;
  for (int i = 0; i < 4; i++) {
    state += 0x9e3779b97f4a7c15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    r->s[i] = z ^ (z >> 31);
  }
}

uint64_t or_rng_next_u64(or_rng *r) {
  uint64_t *s = r->s;
  uint64_t res = rotl64(s[0] + s[3], 23) + s[0];
  uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return res;
}

/* next_u32 takes the upper half of next_u64 (the low bits are the weak ones). */
uint32_t or_rng_next_u32(or_rng *r) { return (uint32_t)(or_rng_next_u64(r) >> 32); }

/* p3-goldilocks StandardUniform: rejection-sample a canonical u64. */
uint64_t or_sample_gl(or_rng *r) {
  for (;;) {
    uint64_t v = or_rng_next_u64(r);
    if (v < OR_GL_P) return v;
  }
}

/* p3-monty-31 StandardUniform: a 31-bit draw (next_u32 >> 1) accepted when < p is
 * taken as the MONTGOMERY form of the element, so the canonical value is v * 2^-32.
 * Parity unpinned: no in-repo vector fixes BabyBear constants. */
uint32_t or_sample_bb(or_rng *r) {
  static uint32_t rinv = 0;
  if (!rinv) rinv = or_bb_inv((uint32_t)((1ull << 32) % OR_BB_P));
  for (;;) {
    uint32_t v = or_rng_next_u32(r) >> 1;
    if (v < OR_BB_P) return or_bb_mul(v, rinv);
  }
}

void or_rng_fill_bb(uint64_t seed, uint32_t *out, size_t n) {
  or_rng r;
  or_rng_seed(&r, seed);
  for (size_t i = 0; i < n; i++) out[i] = or_sample_bb(&r);
}

void or_rng_fill_u64(uint64_t seed, uint64_t *out, size_t n) {
  or_rng r;
  or_rng_seed(&r, seed);
  for (size_t i = 0; i < n; i++) out[i] = or_rng_next_u64(&r);
}

/* ========================================================================== */
/* Poseidon2                                                                   */
/* Structure: zkf-metal/src/shaders/poseidon2.metal:1-154 (Goldilocks),        */
/* :157-264 (BabyBear); zkf-backends/src/wrapping/poseidon2_goldilocks.rs:117-345. */
/* ========================================================================== */

/* poseidon2_round_numbers_128 for D = 7 (p3-poseidon2 0.4.2 table):
 * 31-bit fields: width 16 -> (8, 13), width 24 -> (8, 21);
 * 64-bit fields: widths 8/12/16/20 -> (8, 22). */
int or_p2_round_numbers(int field, int width, int *rounds_f, int *rounds_p) {
  if (field == OR_FIELD_BABYBEAR) {
    if (width == 16) { *rounds_f = 8; *rounds_p = 13; return 0; }
    if (width == 24) { *rounds_f = 8; *rounds_p = 21; return 0; }
    return -1;
  }
  if (width == 8 || width == 12 || width == 16 || width == 20) {
    *rounds_f = 8;
    *rounds_p = 22;
    return 0;
  }
  return -1;
}

/* flatten_round_constants(seed): ExternalLayerConstants::new_from_rng(R_F) draws the
 * R_F/2 initial then R_F/2 terminal width-arrays, then R_P internal draws follow from
 * the same rng.  Layout [initial | internal | terminal]
 * (zkf-metal/src/poseidon2/babybear.rs:76-111, goldilocks.rs:42-83). */
int or_p2_constants_bb(uint64_t seed, int width, uint32_t *flat, size_t cap) {
  int rf, rp;
  if (or_p2_round_numbers(OR_FIELD_BABYBEAR, width, &rf, &rp)) return -1;
  size_t need = (size_t)rf * width + rp;
  if (cap < need) return -1;
  or_rng r;
  or_rng_seed(&r, seed);
  uint32_t *ext = (uint32_t *)malloc(sizeof(uint32_t) * rf * width);
  for (int i = 0; i < rf * width; i++) ext[i] = or_sample_bb(&r);
  size_t half = (size_t)(rf / 2) * width;
  memcpy(flat, ext, half * 4);
  for (int i = 0; i < rp; i++) flat[half + i] = or_sample_bb(&r);
  memcpy(flat + half + rp, ext + half, half * 4);
  free(ext);
  return (int)need;
}

int or_p2_constants_gl(uint64_t seed, int width, uint64_t *flat, size_t cap) {
  int rf, rp;
  if (or_p2_round_numbers(OR_FIELD_GOLDILOCKS, width, &rf, &rp)) return -1;
  size_t need = (size_t)rf * width + rp;
  if (cap < need) return -1;
  or_rng r;
  or_rng_seed(&r, seed);
  uint64_t *ext = (uint64_t *)malloc(sizeof(uint64_t) * rf * width);
  for (int i = 0; i < rf * width; i++) ext[i] = or_sample_gl(&r);
  size_t half = (size_t)(rf / 2) * width;
  memcpy(flat, ext, half * 8);
  for (int i = 0; i < rp; i++) flat[half + i] = or_sample_gl(&r);
  memcpy(flat + half + rp, ext + half, half * 8);
  free(ext);
  return (int)need;
}

/* BabyBear width-16 internal diagonal V =
 * [-2, 1, 2, 1/2, 3, 4, -1/2, -3, -4, 1/2^8, 1/4, 1/8, 1/2^27, -1/2^8, -1/16, -1/2^27]
 * (zkf-metal/src/poseidon2/babybear.rs:14-58). */
void or_p2_diag_bb16(uint32_t out[16]) {
  const uint32_t P = OR_BB_P;
  uint32_t inv2 = or_bb_inv(2);
#define INVP2(e) or_bb_pow(inv2, (e))
  uint32_t v[16] = {P - 2, 1, 2, inv2, 3, 4, P - inv2, P - 3, P - 4,
                    INVP2(8), INVP2(2), INVP2(3), INVP2(27),
                    P - INVP2(8), P - INVP2(4), P - INVP2(27)};
#undef INVP2
  memcpy(out, v, sizeof v);
}

/* MATRIX_DIAG_16_GOLDILOCKS (zkf-metal/src/poseidon2/goldilocks.rs:21-38). */
void or_p2_diag_gl16(uint64_t out[16]) {
  static const uint64_t d[16] = {
      0xde9b91a467d6afc0ull, 0xc5f16b9c76a9be17ull, 0x0ab0fef2d540ac55ull, 0x3001d27009d05773ull,
      0xed23b1f906d3d9ebull, 0x5ce73743cba97054ull, 0x1c3bab944af4ba24ull, 0x2faa105854dbafaeull,
      0x53ffb3ae6d421a10ull, 0xbcda9df8884ba396ull, 0xfc1273e4a31807bbull, 0xc77952573d5142c0ull,
      0x56683339a819b85eull, 0x328fcbd8f0ddc8ebull, 0xb5101e303fce9cb7ull, 0x774487b8c40089bbull};
  memcpy(out, d, sizeof d);
}

/* Goldilocks width-12 internal diagonal.  The reference holds no width-12 instance
 * (its Poseidon2 is width 16 for both fields), so this one is SELF-GENERATED and
 * parity unpinned: twelve draws of the Goldilocks sampler from SmallRng seeded with
 * the ASCII bytes "W12DIAG" (0x57313244494147), each accepted only if it is not 0 or 1
 * and differs from the ones drawn before.  Product and oracle derive it the same way. */
void or_p2_diag_gl12(uint64_t out[12]) {
  or_rng r;
  or_rng_seed(&r, 0x57313244494147ull);
  int k = 0;
  while (k < 12) {
    uint64_t v = or_sample_gl(&r);
    int ok = v > 1;
    for (int j = 0; j < k && ok; j++) ok = out[j] != v;
    if (ok) out[k++] = v;
  }
}

/* External MDS (mds_light_permutation with MDSMat4): M4 = circ-like
 * [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]] on each 4-chunk, then every element adds
 * the sum of its residue class mod 4 (poseidon2_goldilocks.rs:267-321). */
static void p2_ext_mds(int f, uint64_t *s, int w) {
  for (int c = 0; c < w; c += 4) {
    uint64_t a = s[c], b = s[c + 1], x = s[c + 2], y = s[c + 3];
    uint64_t t01 = f_add(f, a, b), t23 = f_add(f, x, y), t0123 = f_add(f, t01, t23);
    uint64_t t01123 = f_add(f, t0123, b), t01233 = f_add(f, t0123, y);
    s[c] = f_add(f, t01123, t01);
    s[c + 1] = f_add(f, t01123, f_add(f, x, x));
    s[c + 2] = f_add(f, t01233, t23);
    s[c + 3] = f_add(f, t01233, f_add(f, a, a));
  }
  uint64_t sums[4] = {0, 0, 0, 0};
  for (int i = 0; i < w; i++) sums[i & 3] = f_add(f, sums[i & 3], s[i]);
  for (int i = 0; i < w; i++) s[i] = f_add(f, s[i], sums[i & 3]);
}

static inline uint64_t p2_sbox(int f, uint64_t x) {
  uint64_t x2 = f_mul(f, x, x), x3 = f_mul(f, x2, x), x4 = f_mul(f, x2, x2);
  return f_mul(f, x4, x3);
}

/* Permutation: initial external MDS; R_F/2 external rounds (add rc, x^7, MDS);
 * R_P internal rounds (rc + x^7 on s[0], then s_i <- d_i s_i + sum); R_F/2 external
 * rounds (poseidon2.metal:92-154, poseidon2_goldilocks.rs:117-140). */
static void p2_permute_one(int f, uint64_t *s, int w, const uint64_t *rc, int rf, int rp,
                           const uint64_t *diag) {
  size_t o = 0;
  p2_ext_mds(f, s, w);
  for (int r = 0; r < rf / 2; r++) {
    for (int i = 0; i < w; i++) s[i] = p2_sbox(f, f_add(f, s[i], rc[o + i]));
    o += w;
    p2_ext_mds(f, s, w);
  }
  for (int r = 0; r < rp; r++) {
    s[0] = p2_sbox(f, f_add(f, s[0], rc[o++]));
    uint64_t sum = 0;
    for (int i = 0; i < w; i++) sum = f_add(f, sum, s[i]);
    for (int i = 0; i < w; i++) s[i] = f_add(f, f_mul(f, s[i], diag[i]), sum);
  }
  for (int r = 0; r < rf / 2; r++) {
    for (int i = 0; i < w; i++) s[i] = p2_sbox(f, f_add(f, s[i], rc[o + i]));
    o += w;
    p2_ext_mds(f, s, w);
  }
}

void or_p2_permute_bb(uint32_t *states, size_t n_states, int width, const uint32_t *rc,
                      int rounds_f, int rounds_p, const uint32_t *diag) {
  size_t nrc = (size_t)rounds_f * width + rounds_p;
  uint64_t *rc64 = (uint64_t *)malloc(8 * nrc), d64[32];
  for (size_t i = 0; i < nrc; i++) rc64[i] = rc[i];
  for (int i = 0; i < width; i++) d64[i] = diag[i];
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n_states; k++) {
    uint64_t s[32];
    for (int i = 0; i < width; i++) s[i] = states[k * width + i];
    p2_permute_one(OR_FIELD_BABYBEAR, s, width, rc64, rounds_f, rounds_p, d64);
    for (int i = 0; i < width; i++) states[k * width + i] = (uint32_t)s[i];
  }
  free(rc64);
}

void or_p2_permute_gl(uint64_t *states, size_t n_states, int width, const uint64_t *rc,
                      int rounds_f, int rounds_p, const uint64_t *diag) {
#pragma omp parallel for schedule(static)
  for (size_t k = 0; k < n_states; k++)
    p2_permute_one(OR_FIELD_GOLDILOCKS, states + k * width, width, rc, rounds_f, rounds_p, diag);
}

/* ========================================================================== */
/* Hasher: PaddingFreeSponge<Perm, W, 8, OUT> + TruncatedPermutation<Perm,2,OUT,W> */
/* (zkf-backends/src/plonky3.rs:55-56; poseidon2_goldilocks.rs:373-415)          */
/* ========================================================================== */

int or_hasher_init(or_hasher *h, int field, int width, uint64_t seed) {
  memset(h, 0, sizeof *h);
  h->field = field;
  h->width = width;
  h->rate = 8;
  h->out = width == 16 ? 8 : (width == 12 ? 4 : 0);
  if (!h->out) return -1;
  if (or_p2_round_numbers(field, width, &h->rounds_f, &h->rounds_p)) return -1;
  if (field == OR_FIELD_BABYBEAR) {
    uint32_t rc[512], d[16];
    int n = or_p2_constants_bb(seed, width, rc, 512);
    if (n < 0 || width != 16) return -1;
    for (int i = 0; i < n; i++) h->rc[i] = rc[i];
    or_p2_diag_bb16(d);
    for (int i = 0; i < 16; i++) h->diag[i] = d[i];
  } else {
    if (or_p2_constants_gl(seed, width, h->rc, 512) < 0) return -1;
    if (width == 16)
      or_p2_diag_gl16(h->diag);
    else
      or_p2_diag_gl12(h->diag);
  }
  return 0;
}

static void hasher_perm(const or_hasher *h, uint64_t *s) {
  p2_permute_one(h->field, s, h->width, h->rc, h->rounds_f, h->rounds_p, h->diag);
}

/* Overwrite-mode sponge: absorb RATE elements into s[0..RATE) and permute; a partial
 * final chunk overwrites only its own positions, then permutes; an empty final chunk
 * does not permute.  Digest = s[0..OUT). */
typedef struct {
  uint64_t s[32];
  int pos;
} sponge_t;
static inline void sponge_absorb(const or_hasher *h, sponge_t *sp, uint64_t v) {
  sp->s[sp->pos++] = v;
  if (sp->pos == h->rate) {
    hasher_perm(h, sp->s);
    sp->pos = 0;
  }
}
static inline void sponge_finish(const or_hasher *h, sponge_t *sp, uint64_t *dig) {
  if (sp->pos) hasher_perm(h, sp->s);
  for (int i = 0; i < h->out; i++) dig[i] = sp->s[i];
}

void or_sponge(const or_hasher *h, const void *elems, size_t n, void *digest_out) {
  sponge_t sp;
  memset(&sp, 0, sizeof sp);
  for (size_t i = 0; i < n; i++) sponge_absorb(h, &sp, ld(h->field, elems, i));
  uint64_t d[16];
  sponge_finish(h, &sp, d);
  for (int i = 0; i < h->out; i++) st(h->field, digest_out, i, d[i]);
}

static void compress64(const or_hasher *h, const uint64_t *l, const uint64_t *r, uint64_t *o) {
  uint64_t s[32];
  memset(s, 0, sizeof s);
  for (int i = 0; i < h->out; i++) {
    s[i] = l[i];
    s[h->out + i] = r[i];
  }
  hasher_perm(h, s);
  for (int i = 0; i < h->out; i++) o[i] = s[i];
}

void or_compress(const or_hasher *h, const void *left, const void *right, void *out) {
  uint64_t l[16], r[16], o[16];
  for (int i = 0; i < h->out; i++) {
    l[i] = ld(h->field, left, i);
    r[i] = ld(h->field, right, i);
  }
  compress64(h, l, r, o);
  for (int i = 0; i < h->out; i++) st(h->field, out, i, o[i]);
}

/* Digest of one row index across several matrices (hash_iter over the flat_map of
 * the rows, vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:244-262). */
static void hash_row_multi(const or_hasher *h, const void *const *mats, const size_t *widths,
                           size_t n_mats, size_t row, uint64_t *dig) {
  sponge_t sp;
  memset(&sp, 0, sizeof sp);
  for (size_t m = 0; m < n_mats; m++)
    for (size_t c = 0; c < widths[m]; c++)
      sponge_absorb(h, &sp, ld(h->field, mats[m], row * widths[m] + c));
  sponge_finish(h, &sp, dig);
}

void or_hash_rows(const or_hasher *hs, const void *const *mats, const size_t *widths,
                  size_t n_mats, size_t height, void *digests) {
#pragma omp parallel for schedule(static)
  for (size_t r = 0; r < height; r++) {
    uint64_t d[16];
    hash_row_multi(hs, mats, widths, n_mats, r, d);
    for (int i = 0; i < hs->out; i++) st(hs->field, digests, r * hs->out + i, d[i]);
  }
}

/* ========================================================================== */
/* MMCS: p3 MerkleTree::new (vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:84-151),   */
/* first_digest_layer (:202-266), compress_and_inject (:272-350), compress (:359-403) */
/* ========================================================================== */

static size_t next_pow2(size_t x) {
  size_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

size_t or_mmcs_layers_total(size_t max_height) {
  size_t len = max_height == 1 ? 1 : max_height + (max_height & 1), tot = len;
  while (len > 1) {
    len = len == 2 ? 1 : ((len / 2 + 1) & ~(size_t)1);
    tot += len;
  }
  return tot;
}

int or_mmcs_commit(const or_hasher *h, const void *const *mats, const size_t *heights,
                   const size_t *widths, size_t n_mats, void *layers_out, size_t layers_cap,
                   size_t *layer_lens, int max_layers) {
  if (n_mats == 0) return -1;
  const int D = h->out;
  const int f = h->field;
  /* stable sort of matrix indices by height, tallest first */
  size_t *ord = (size_t *)malloc(sizeof(size_t) * n_mats);
  for (size_t i = 0; i < n_mats; i++) ord[i] = i;
  for (size_t i = 1; i < n_mats; i++) {
    size_t k = ord[i], j = i;
    while (j > 0 && heights[ord[j - 1]] < heights[k]) {
      ord[j] = ord[j - 1];
      j--;
    }
    ord[j] = k;
  }
  for (size_t i = 0; i + 1 < n_mats; i++) {
    size_t a = heights[ord[i]], b = heights[ord[i + 1]];
    if (a != b && next_pow2(a) == next_pow2(b)) {
      free(ord);
      return -1;
    }
  }
  size_t max_h = heights[ord[0]];
  if (max_h == 0) {
    free(ord);
    return -1;
  }
  if (or_mmcs_layers_total(max_h) * D > layers_cap) {
    free(ord);
    return -1;
  }
  /* group of tallest matrices */
  size_t ng = 0;
  while (ng < n_mats && heights[ord[ng]] == max_h) ng++;
  const void **gm = (const void **)malloc(sizeof(void *) * n_mats);
  size_t *gw = (size_t *)malloc(sizeof(size_t) * n_mats);
  for (size_t i = 0; i < ng; i++) {
    gm[i] = mats[ord[i]];
    gw[i] = widths[ord[i]];
  }
  size_t len0 = max_h == 1 ? 1 : max_h + (max_h & 1);
  uint64_t *prev = (uint64_t *)calloc(len0 * D, 8);
#pragma omp parallel for schedule(static)
  for (size_t r = 0; r < max_h; r++) hash_row_multi(h, gm, gw, ng, r, prev + r * D);
  size_t prev_len = len0, off = 0;
  int nl = 0;
  for (size_t i = 0; i < prev_len * D; i++) st(f, layers_out, off + i, prev[i]);
  off += prev_len * D;
  layer_lens[nl++] = prev_len;
  size_t next_m = ng;
  while (prev_len > 1) {
    if (nl >= max_layers) {
      nl = -1;
      break;
    }
    size_t next_layer_len = next_pow2(prev_len / 2);
    size_t ni = 0;
    while (next_m + ni < n_mats && next_pow2(heights[ord[next_m + ni]]) == next_layer_len) ni++;
    size_t half = prev_len / 2;
    size_t padded = prev_len == 2 ? 1 : ((half + 1) & ~(size_t)1);
    uint64_t *next = (uint64_t *)calloc(padded * D, 8);
    size_t inj_h = ni ? heights[ord[next_m]] : 0;
    for (size_t i = 0; i < ni; i++) {
      gm[i] = mats[ord[next_m + i]];
      gw[i] = widths[ord[next_m + i]];
    }
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < half; i++) {
      uint64_t c[16];
      compress64(h, prev + 2 * i * D, prev + (2 * i + 1) * D, c);
      if (ni) {
        uint64_t rd[16] = {0};
        if (i < inj_h) hash_row_multi(h, gm, gw, ni, i, rd);
        compress64(h, c, rd, next + i * D);
      } else {
        memcpy(next + i * D, c, 8 * D);
      }
    }
    next_m += ni;
    free(prev);
    prev = next;
    prev_len = padded;
    for (size_t i = 0; i < prev_len * D; i++) st(f, layers_out, off + i, prev[i]);
    off += prev_len * D;
    layer_lens[nl++] = prev_len;
  }
  free(prev);
  free(gm);
  free(gw);
  free(ord);
  return nl;
}

/* ========================================================================== */
/* DFT: column-wise radix-2 DIT after a bit-reversal, twiddle g^(j*n/(2*half)),  */
/* inverse with g^-1 and a 1/n scale (zkf-metal/src/ntt/p3_adapter.rs:462-572).  */
/* ========================================================================== */

static inline size_t rev_bits(size_t x, int bits) {
  size_t r = 0;
  for (int i = 0; i < bits; i++) {
    r = (r << 1) | (x & 1);
    x >>= 1;
  }
  return r;
}

static void dft_column(int f, uint64_t *col, int log_n, const uint64_t *pw, int inverse,
                       uint64_t n_inv) {
  size_t n = (size_t)1 << log_n;
  for (size_t i = 0; i < n; i++) {
    size_t j = rev_bits(i, log_n);
    if (i < j) {
      uint64_t t = col[i];
      col[i] = col[j];
      col[j] = t;
    }
  }
  for (int stage = 0; stage < log_n; stage++) {
    size_t half = (size_t)1 << stage, step = n >> (stage + 1);
    for (size_t g = 0; g < n; g += 2 * half)
      for (size_t j = 0; j < half; j++) {
        uint64_t w = pw[j * step];
        uint64_t a = col[g + j], b = f_mul(f, w, col[g + j + half]);
        col[g + j] = f_add(f, a, b);
        col[g + j + half] = f_sub(f, a, b);
      }
  }
  if (inverse)
    for (size_t i = 0; i < n; i++) col[i] = f_mul(f, col[i], n_inv);
}

void or_dft_batch(int field, void *mat, int log_h, size_t w, int inverse) {
  size_t n = (size_t)1 << log_h;
  if (w == 0) return;
  uint64_t g = or_two_adic_generator(field, log_h);
  if (inverse) g = f_inv(field, g);
  uint64_t *pw = (uint64_t *)malloc(8 * (n / 2 + 1));
  pw[0] = 1;
  for (size_t i = 1; i <= n / 2; i++) pw[i] = f_mul(field, pw[i - 1], g);
  uint64_t n_inv = f_inv(field, n % f_modulus(field));
#pragma omp parallel
  {
    uint64_t *col = (uint64_t *)malloc(8 * n);
#pragma omp for schedule(dynamic)
    for (size_t c = 0; c < w; c++) {
      for (size_t r = 0; r < n; r++) col[r] = ld(field, mat, r * w + c);
      dft_column(field, col, log_h, pw, inverse, n_inv);
      for (size_t r = 0; r < n; r++) st(field, mat, r * w + c, col[r]);
    }
    free(col);
  }
  free(pw);
}

void or_bit_reverse_rows(int field, void *mat, int log_h, size_t w) {
  size_t n = (size_t)1 << log_h, es = f_esize(field);
  char *m = (char *)mat, *tmp = (char *)malloc(es * w);
  for (size_t i = 0; i < n; i++) {
    size_t j = rev_bits(i, log_h);
    if (i < j) {
      memcpy(tmp, m + i * w * es, w * es);
      memcpy(m + i * w * es, m + j * w * es, w * es);
      memcpy(m + j * w * es, tmp, w * es);
    }
  }
  free(tmp);
}

/* p3-dft 0.4.2 default coset_lde_batch: idft_batch, zero-extend to 2^added_bits times
 * the height, multiply row i by shift^i (coset_dft_batch), dft_batch.  The PCS then
 * bit-reverses the rows (TwoAdicFriPcs::commit; LDE row i <-> x = shift * g^rev(i),
 * zkf-backends/src/wrapping/stark_to_groth16.rs:2324-2346). */
void or_coset_lde_batch(int field, const void *trace, int log_h, size_t w, int log_blowup,
                        uint64_t shift, int bitrev, void *out) {
  size_t n = (size_t)1 << log_h, es = f_esize(field);
  size_t N = n << log_blowup;
  void *coef = malloc(n * w * es);
  memcpy(coef, trace, n * w * es);
  or_dft_batch(field, coef, log_h, w, 1);
  memset(out, 0, N * w * es);
  uint64_t sp = 1;
  for (size_t r = 0; r < n; r++) {
    for (size_t c = 0; c < w; c++)
      st(field, out, r * w + c, f_mul(field, ld(field, coef, r * w + c), sp));
    sp = f_mul(field, sp, shift);
  }
  free(coef);
  or_dft_batch(field, out, log_h + log_blowup, w, 0);
  if (bitrev) or_bit_reverse_rows(field, out, log_h + log_blowup, w);
}

/* ========================================================================== */
/* FRI                                                                         */
/* ========================================================================== */

/* FriAccelerator::fold_* and the Metal kernels (zkf-metal/src/shaders/fri.metal:14-53,
 * zkf-core/src/acceleration.rs:197-217, zkf-metal/src/fri.rs:187-198). */
void or_fri_fold_base(int field, const void *evals, size_t n_out, uint64_t alpha,
                      const void *inv_tw, void *out) {
  uint64_t inv2 = f_inv(field, 2);
  for (size_t i = 0; i < n_out; i++) {
    uint64_t e = ld(field, evals, 2 * i), o = ld(field, evals, 2 * i + 1);
    uint64_t s = f_mul(field, f_add(field, e, o), inv2);
    uint64_t d = f_mul(field, f_mul(field, f_sub(field, e, o), ld(field, inv_tw, i)), alpha);
    st(field, out, i, f_add(field, s, d));
  }
}

void or_fri_inv_twiddles(int field, size_t n_out, void *out) {
  int log_n = 0;
  while (((size_t)1 << log_n) < n_out) log_n++;
  uint64_t g_inv = f_inv(field, or_two_adic_generator(field, log_n + 1));
  uint64_t inv2 = f_inv(field, 2);
  uint64_t p = inv2;
  for (size_t i = 0; i < n_out; i++) {
    st(field, out, rev_bits(i, log_n), p);
    p = f_mul(field, p, g_inv);
  }
}

/* BabyBear quartic extension F[x]/(x^4 - 11) (p3-baby-bear BinomiallyExtendable<4>,
 * W = 11; parity unpinned in-repo: the reference FRI runs over the base field). */
void or_bb4_mul(const uint32_t *a, const uint32_t *b, uint32_t *o) {
  uint64_t c[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) c[i + j] = or_bb_add((uint32_t)c[i + j], or_bb_mul(a[i], b[j]));
  for (int k = 0; k < 4; k++) {
    uint32_t hi = k + 4 < 7 ? (uint32_t)c[k + 4] : 0;
    o[k] = or_bb_add((uint32_t)c[k], or_bb_mul(11, hi));
  }
}

/* p3 TwoAdicFriFolding::fold_matrix for arity 2: with g = two_adic_generator(log n_out + 1),
 * result[i] = (1/2 + beta/2 * g^-rev(i)) r0 + (1/2 - beta/2 * g^-rev(i)) r1,
 * where (r0, r1) = (evals[2i], evals[2i+1]) are the values at +x and -x. */
void or_fri_fold_ext4(const uint32_t *evals, size_t n_out, const uint32_t beta[4],
                      uint32_t *out) {
  int log_n = 0;
  while (((size_t)1 << log_n) < n_out) log_n++;
  uint32_t g_inv = or_bb_inv((uint32_t)or_two_adic_generator(OR_FIELD_BABYBEAR, log_n + 1));
  uint32_t inv2 = or_bb_inv(2);
  uint32_t *pows = (uint32_t *)malloc(4 * n_out);
  uint32_t p = 1;
  for (size_t i = 0; i < n_out; i++) {
    pows[rev_bits(i, log_n)] = p;
    p = or_bb_mul(p, g_inv);
  }
  uint32_t hb[4];
  for (int k = 0; k < 4; k++) hb[k] = or_bb_mul(beta[k], inv2);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n_out; i++) {
    const uint32_t *r0 = evals + 8 * i, *r1 = evals + 8 * i + 4;
    uint32_t pw[4], lo[4], hi[4], a[4], b[4];
    for (int k = 0; k < 4; k++) pw[k] = or_bb_mul(hb[k], pows[i]);
    for (int k = 0; k < 4; k++) {
      lo[k] = or_bb_add(k == 0 ? inv2 : 0, pw[k]);
      hi[k] = or_bb_sub(k == 0 ? inv2 : 0, pw[k]);
    }
    or_bb4_mul(lo, r0, a);
    or_bb4_mul(hi, r1, b);
    for (int k = 0; k < 4; k++) out[4 * i + k] = or_bb_add(a[k], b[k]);
  }
  free(pows);
}

/* out[i] = sum_j alpha^j * lde[i][j] in BabyBear^4: the alpha-reduction of committed
 * columns into one extension codeword (p3-fri 0.4.2 open, without the (x - z) quotient). */
void or_combine_columns_ext4(const uint32_t *lde, size_t rows, size_t width, const uint32_t alpha[4],
                             uint32_t *out) {
  uint32_t *pw = (uint32_t *)malloc(16 * (width ? width : 1));
  uint32_t cur[4] = {1, 0, 0, 0};
  for (size_t j = 0; j < width; j++) {
    memcpy(pw + 4 * j, cur, 16);
    uint32_t nx[4];
    or_bb4_mul(cur, alpha, nx);
    memcpy(cur, nx, 16);
  }
#pragma omp parallel for schedule(static)
  for (size_t r = 0; r < rows; r++) {
    uint32_t acc[4] = {0, 0, 0, 0};
    for (size_t j = 0; j < width; j++)
      for (int k = 0; k < 4; k++) acc[k] = or_bb_add(acc[k], or_bb_mul(lde[r * width + j], pw[4 * j + k]));
    memcpy(out + 4 * r, acc, 16);
  }
  free(pw);
}

int or_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
