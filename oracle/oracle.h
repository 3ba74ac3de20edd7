/*
 * oracle.h — CPU restatement of the ZirOS / Plonky3 polynomial-commitment path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * product in ziros_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it; the product
 * never links or calls it.
 *
 * Parity anchors (see the per-function comments in oracle.c for file:line):
 *   - Goldilocks Poseidon2 W16 seed 42 golden vector
 *     (zkf-backends/src/wrapping/poseidon2_goldilocks.rs:546-563) — PINNED.
 *   - DFT([1,2,3,4])[0] = 10 (zkf-metal/src/ntt/p3_adapter.rs:605-619) — PINNED.
 *   - BabyBear Poseidon2 constants (p3-monty-31 sampler), the BabyBear
 *     quartic extension (x^4 - 11) and Goldilocks width-12 — parity unpinned:
 *     no in-repo vector fixes them; restated from the published Plonky3 0.4.2
 *     algorithms and labelled as such.
 *
 * Every field value crossing this interface is canonical (in [0, p)).
 */
#ifndef ZKB_ORACLE_H
#define ZKB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_FIELD_BABYBEAR 0
#define OR_FIELD_GOLDILOCKS 1

#define OR_BB_P 0x78000001u
#define OR_GL_P 0xFFFFFFFF00000001ull

/* ---- scalar field ops (canonical in/out) ---- */
uint32_t or_bb_add(uint32_t a, uint32_t b);
uint32_t or_bb_sub(uint32_t a, uint32_t b);
uint32_t or_bb_mul(uint32_t a, uint32_t b);
uint32_t or_bb_pow(uint32_t a, uint64_t e);
uint32_t or_bb_inv(uint32_t a);
uint64_t or_gl_add(uint64_t a, uint64_t b);
uint64_t or_gl_sub(uint64_t a, uint64_t b);
uint64_t or_gl_mul(uint64_t a, uint64_t b);
uint64_t or_gl_pow(uint64_t a, uint64_t e);
uint64_t or_gl_inv(uint64_t a);
uint64_t or_two_adic_generator(int field, int bits);
uint64_t or_field_generator(int field);

/* ---- rand 0.9 SmallRng (xoshiro256++ seeded through SplitMix64) ---- */
typedef struct { uint64_t s[4]; } or_rng;
void or_rng_seed(or_rng *r, uint64_t seed);
uint64_t or_rng_next_u64(or_rng *r);
uint32_t or_rng_next_u32(or_rng *r);
uint64_t or_sample_gl(or_rng *r);
uint32_t or_sample_bb(or_rng *r);
/* Fill `out` with `n` draws; returns final rng state in *r. */
void or_rng_fill_u64(uint64_t seed, uint64_t *out, size_t n);
void or_rng_fill_bb(uint64_t seed, uint32_t *out, size_t n);

/* ---- Poseidon2 ---- */
int or_p2_round_numbers(int field, int width, int *rounds_f, int *rounds_p);
/* Flat constants [ext_initial (rf/2*w) | internal (rp) | ext_terminal (rf/2*w)] */
int or_p2_constants_bb(uint64_t seed, int width, uint32_t *flat, size_t cap);
int or_p2_constants_gl(uint64_t seed, int width, uint64_t *flat, size_t cap);
void or_p2_diag_bb16(uint32_t out[16]);
void or_p2_diag_gl16(uint64_t out[16]);
void or_p2_diag_gl12(uint64_t out[12]);
/* In-place batch permutation over n_states states of `width` elements. */
void or_p2_permute_bb(uint32_t *states, size_t n_states, int width, const uint32_t *rc,
                      int rounds_f, int rounds_p, const uint32_t *diag);
void or_p2_permute_gl(uint64_t *states, size_t n_states, int width, const uint64_t *rc,
                      int rounds_f, int rounds_p, const uint64_t *diag);

/* ---- hashing configuration: one Poseidon2 instance + sponge geometry ---- */
typedef struct {
  int field;     /* OR_FIELD_* */
  int width;     /* permutation width (16, or 12 for Goldilocks) */
  int rate;      /* sponge rate (8) */
  int out;       /* digest elements (8 for W16, 4 for W12) */
  int rounds_f, rounds_p;
  uint64_t rc[512];
  uint64_t diag[16];
} or_hasher;
int or_hasher_init(or_hasher *h, int field, int width, uint64_t seed);
/* PaddingFreeSponge<Perm, W, RATE, OUT>::hash_iter on `n` elements (u32 or u64). */
void or_sponge(const or_hasher *h, const void *elems, size_t n, void *digest_out);
/* TruncatedPermutation<Perm, 2, OUT, W>::compress */
void or_compress(const or_hasher *h, const void *left, const void *right, void *out);
/* Hash each row of one or more equal-height row-major matrices into digests.
 * mats[i] points to an h x widths[i] matrix; digests: h * out elements. */
void or_hash_rows(const or_hasher *hs, const void *const *mats, const size_t *widths,
                  size_t n_mats, size_t height, void *digests);

/* ---- MMCS (p3-merkle-tree semantics) ----
 * Matrices are row-major; element size follows the field.  Layers are written
 * back-to-back into `layers_out` (digest elements); layer_lens[i] receives the
 * number of digests of layer i.  Returns the number of layers, or -1 on error.
 */
int or_mmcs_commit(const or_hasher *h, const void *const *mats, const size_t *heights,
                   const size_t *widths, size_t n_mats, void *layers_out, size_t layers_cap,
                   size_t *layer_lens, int max_layers);
size_t or_mmcs_layers_total(size_t max_height);

/* ---- DFT / LDE (column-wise on row-major h x w) ---- */
void or_dft_batch(int field, void *mat, int log_h, size_t w, int inverse);
/* p3 coset_lde_batch(mat, log_blowup, shift) followed by bit_reverse_rows when bitrev. */
void or_coset_lde_batch(int field, const void *trace, int log_h, size_t w, int log_blowup,
                        uint64_t shift, int bitrev, void *out);
void or_bit_reverse_rows(int field, void *mat, int log_h, size_t w);

/* ---- FRI ---- */
/* FriAccelerator::fold_* semantics:
 * g[i] = (f[2i] + f[2i+1]) / 2 + alpha * (f[2i] - f[2i+1]) * inv_tw[i] */
void or_fri_fold_base(int field, const void *evals, size_t n_out, uint64_t alpha,
                      const void *inv_tw, void *out);
/* p3 TwoAdicFriFolding::fold_matrix for the BabyBear quartic extension.
 * evals: 2*n_out EF elements (4 u32 each), bit-reversed domain order. */
void or_fri_fold_ext4(const uint32_t *evals, size_t n_out, const uint32_t beta[4],
                      uint32_t *out);
/* Inverse twiddles that make or_fri_fold_base equal p3 fold_matrix:
 * inv_tw[i] = g_inv^{rev(i)} / 2, g = two_adic_generator(log2(n_out)+1). */
void or_fri_inv_twiddles(int field, size_t n_out, void *out);
void or_bb4_mul(const uint32_t *a, const uint32_t *b, uint32_t *out);
void or_combine_columns_ext4(const uint32_t *lde, size_t rows, size_t width, const uint32_t alpha[4],
                             uint32_t *out);

/* ---- timing helper for the CPU baseline ---- */
int or_num_threads(void);
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
