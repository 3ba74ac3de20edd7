/*
 * zkb200.h — C ABI of the B200 polynomial-commitment library (libzkb200.so).
 *
 * The library is a drop-in for the ZirOS accelerator path of the Plonky3 STARK
 * backend: coset NTT / low-degree extension, Poseidon2 Merkle commitment (MMCS)
 * and FRI folding over BabyBear and Goldilocks.  Each entry point names the
 * reference interface it replaces (paths relative to the ZirOS repository root).
 *
 * Conventions
 *  - Field elements are canonical integers in [0, p): uint32_t for BabyBear,
 *    uint64_t for Goldilocks.  Matrices are row-major (p3 RowMajorMatrix).
 *  - Return status: ZKB_OK (0); ZKB_DECLINED (1) = "not accelerated, use the CPU
 *    path" (the reference's `false` / `None`, e.g. zkf-metal/src/poseidon2/mod.rs:44-46);
 *    negative = error.  The message of the last failure on the calling thread is
 *    returned by zkb_last_error_message(), as zkf-ffi does
 *    (zkf-ffi/src/lib.rs:49-60,165-171).
 *  - Entry points without a suffix take HOST pointers and synchronise before
 *    returning.  `_dev` entry points take DEVICE pointers and a cudaStream_t
 *    (passed as void*; NULL is the CUDA default stream, as in any CUDA API) and
 *    are asynchronous with respect to the host, except where a result is returned
 *    in host memory (roots), which synchronises that stream.
 *  - All entry points are thread-safe.
 */
#ifndef ZKB200_H
#define ZKB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define ZKB_API __attribute__((visibility("default")))
#else
#define ZKB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ZKB_OK 0
#define ZKB_DECLINED 1
#define ZKB_ERR_INVALID (-1)
#define ZKB_ERR_CUDA (-2)
#define ZKB_ERR_OOM (-3)
#define ZKB_ERR_UNSUPPORTED (-4)
#define ZKB_ERR_INTERNAL (-5)
#define ZKB_ERR_TIMEOUT (-6)
#define ZKB_ERR_CANCELLED (-7)

#define ZKB_FIELD_BABYBEAR 0
#define ZKB_FIELD_GOLDILOCKS 1

/* ------------------------------------------------------------------ general */
/* Library version string. */
ZKB_API const char *zkb_version(void);
/* Thread-local message of the last failed call (zkf-ffi zkf_last_error_message,
 * zkf-ffi/src/lib.rs:165-171). */
ZKB_API const char *zkb_last_error_message(void);
/* Number of CUDA devices; 0 when no usable device (MetalContext availability,
 * zkf-metal/src/device.rs:1469-1493). */
ZKB_API int zkb_device_count(void);
/* Select the device used by this thread's subsequent calls. */
ZKB_API int zkb_set_device(int device);

/* Failure detection, after the reference's watchdog and circuit breaker
 * (zkf-metal/src/async_dispatch.rs:16-71,162-204; device.rs:649-662): every host wait
 * on device work has a deadline (env ZKB_WATCHDOG_MS, default 120000; 0 = none).  A
 * device error or an expired deadline opens a process-wide circuit; while it is open,
 * every compute entry point declines (ZKB_DECLINED: the caller takes its CPU path).
 * ZKB_DISABLE=1 declines everything (kill switch, like the reference's ZKF_METAL). */
ZKB_API int zkb_circuit_open(char *why_out, size_t cap);  /* 1 open (reason copied), 0 closed */
ZKB_API void zkb_circuit_reset(void);
/* Fallback thresholds, the reference's ThresholdConfig (zkf-metal/src/tuning.rs:84-111)
 * with its runtime override (tuning.rs:284-300): the host-pointer entry points decline
 * (ZKB_DECLINED, "below threshold") for transforms of fewer rows than `ntt`, batches of
 * fewer permutations than `poseidon2`, trees of fewer leaves than `merkle` and folds of
 * fewer outputs than `fri`, so the caller runs its CPU path.  Default: no minimum, or
 * env ZKB_THRESHOLDS="ntt=4096,poseidon2=1000,merkle=2048,fri=1024".  NULL resets to no
 * minimum.  Device-pointer entry points never decline on size. */
typedef struct {
  uint64_t ntt, poseidon2, merkle, fri;
} zkb_thresholds;
ZKB_API int zkb_set_thresholds(const zkb_thresholds *thresholds);
ZKB_API int zkb_get_thresholds(zkb_thresholds *thresholds_out);
/* Host-side fault injection for tests; nothing is injected on the device.  kind 1: the
 * next `count` device allocations fail as out of memory; kind 2: the next `count` stream
 * waits report an expired deadline (after the work has finished). */
ZKB_API int zkb_debug_inject_fault(int kind, int count);
/* Number of device allocations (stream-ordered pool or cudaMalloc) the library has
 * made in this process.  Tests read it around a call to check that the call allocated
 * nothing.  No counterpart in the reference. */
ZKB_API uint64_t zkb_debug_device_allocations(void);
/* Of those, the allocations of 1 MiB or more (the sizes the library caches) that found no
 * freed block of their size in its cache and took new memory from the stream-ordered pool
 * (which grows, mapping fresh memory, when it has none free).  The bench reads it around its timed region.  No counterpart in
 * the reference. */
ZKB_API uint64_t zkb_debug_pool_allocations(void);
/* Device memory the library keeps for reuse on the current device — freed blocks it caches
 * for allocations of the same size, and the stream-ordered pool's unused memory — goes
 * back to the device, e.g. before a large cudaMalloc of the caller's.  zkb_batch_create
 * does this itself.  No counterpart in the reference. */
ZKB_API int zkb_release_cached_memory(void);

/* Kernel timing.  zkb_profile_start() enables per-launch CUDA events (recorded on
 * the stream each kernel is launched on) and clears earlier records;
 * zkb_profile_stop() disables them, waits for the events and writes one entry per
 * kernel name (at most `cap`); returns the number of names.  This is the per-stage
 * timing hook of the reference's GPU telemetry (zkf-runtime/src/telemetry.rs:1-25,
 * zkf-backends/src/plonky3.rs:806-971). */
typedef struct {
  char name[48];
  uint64_t launches;
  double total_ms;
  double max_ms;
} zkb_kernel_stat;
ZKB_API int zkb_profile_start(void);
ZKB_API int zkb_profile_stop(zkb_kernel_stat *out, int cap);

/* Measured field-multiplication ceiling of the current device: field
 * multiplications per second of independent multiply chains on every SM (the
 * integer-pipe roofline of the Poseidon2 kernels).  No reference counterpart: it
 * is this library's measurement hook. */
ZKB_API int zkb_measure_mul_peak(int field, double *mul_per_s);

/* ---------------------------------------------------------------- Poseidon2 */
/* flatten_round_constants(seed) (zkf-metal/src/poseidon2/babybear.rs:76-111,
 * goldilocks.rs:42-83).  Writes up to `cap` canonical constants in the layout
 * [external initial | internal | external terminal]; returns the count (>0) or <0. */
ZKB_API int zkb_poseidon2_babybear_round_constants(uint64_t seed, uint32_t *out, size_t cap,
                                           uint32_t *n_external_rounds,
                                           uint32_t *n_internal_rounds);
ZKB_API int zkb_poseidon2_goldilocks_round_constants(uint64_t seed, uint32_t width, uint64_t *out,
                                             size_t cap, uint32_t *n_external_rounds,
                                             uint32_t *n_internal_rounds);

/* Poseidon2Accelerator::batch_permute_babybear (zkf-core/src/acceleration.rs:113-145;
 * MetalPoseidon2::batch_permute_babybear, zkf-metal/src/poseidon2/mod.rs:150-257).
 * In-place width-16 permutations of n_elems/16 states. */
ZKB_API int zkb_poseidon2_babybear_permute(uint32_t *states, size_t n_elems, const uint32_t *round_constants,
                                   size_t n_rc, uint32_t n_external_rounds,
                                   uint32_t n_internal_rounds);
/* Poseidon2Accelerator::batch_permute_goldilocks (acceleration.rs:113-145;
 * MetalPoseidon2::batch_permute_goldilocks, poseidon2/mod.rs:36-148).  Width 16. */
ZKB_API int zkb_poseidon2_goldilocks_permute(uint64_t *states, size_t n_elems,
                                     const uint64_t *round_constants, size_t n_rc,
                                     uint32_t n_external_rounds, uint32_t n_internal_rounds);
/* Device-pointer forms of the two permutations above. */
ZKB_API int zkb_poseidon2_babybear_permute_dev(uint32_t *d_states, size_t n_elems,
                                       const uint32_t *round_constants, size_t n_rc,
                                       uint32_t n_external_rounds, uint32_t n_internal_rounds,
                                       void *stream);
ZKB_API int zkb_poseidon2_goldilocks_permute_dev(uint64_t *d_states, size_t n_elems,
                                         const uint64_t *round_constants, size_t n_rc,
                                         uint32_t n_external_rounds, uint32_t n_internal_rounds,
                                         void *stream);

/* ---------------------------------------------------------------------- DFT */
/* TwoAdicSubgroupDft::dft_batch / MetalDft::idft_batch
 * (zkf-metal/src/ntt/p3_adapter.rs:69-106,426-459): column-wise DFT of a row-major
 * 2^log_h x width matrix, natural order in and out, in place.  inverse=1 applies
 * g^-1 twiddles and the 1/n scale. */
ZKB_API int zkb_dft_batch(int field, void *rowmajor, uint32_t log_h, uint32_t width, int inverse);
ZKB_API int zkb_dft_batch_dev(int field, void *d_rowmajor, uint32_t log_h, uint32_t width, int inverse,
                      void *stream);

/* Allocation-free form of zkb_dft_batch_dev, for callers that cannot call cudaMalloc
 * (device memory owned by another allocator, or a path that must not pay the
 * synchronisation an allocation or free can cause).  No counterpart in the reference.
 * Its scratch is a fixed 16 MiB device array held by the library on every GPU that
 * loads it; it must fit the twiddle table plus a copy of the matrix:
 * 2^log_h * elem_bytes (rounded up to 256) + 2^log_h * width * elem_bytes <= 16 MiB,
 * else ZKB_ERR_INVALID with a message.  The first call on a device looks up the
 * array's device address (set-up, once per device); make that first call before any
 * stream capture.  All calls share the array and it keeps the last call's contents
 * (nothing in it needs to start at zero); calls that overlap on the GPU race, so issue
 * them on one stream. */
ZKB_API int zkb_dft_batch_noalloc_dev(int field, void *d_rowmajor, uint32_t log_h, uint32_t width,
                                      int inverse, void *stream);

/* Tile loads of the NTT passes and the fused LDE middle (DFT, LDE, commits;
 * process-wide): 1 = one tensor copy (TMA, cp.async.bulk.tensor into the CTA's own shared memory) of each
 * tile into shared memory (the default), used where the row stride and the column chunk
 * are multiples of 16 bytes (BabyBear: width a multiple of 4, chunks of 4 columns or more;
 * Goldilocks: even width, chunks of 4 or 8; other tiles keep the loads); 0 = coalesced
 * loads straight into registers.  ZKB_NTT_TMA=0 in the environment selects 0 at load.
 * Results are the same bit for bit.  No counterpart in the reference. */
ZKB_API int zkb_set_ntt_tile_loads(int mode);
/* Tensor-copy waits of the NTT tiles that gave up (bounded polls) since the last call;
 * nonzero means those outputs are invalid.  Resets the count. */
ZKB_API int zkb_ntt_tile_load_errors(uint32_t *count);

/* p3 coset_lde_batch(trace, log_blowup, shift) followed, when bitrev_rows=1, by
 * bit_reverse_rows — the LDE that TwoAdicFriPcs::commit hands to the MMCS
 * (zkf-backends/src/plonky3.rs:250-262 -> p3-dft 0.4.2;
 * zkf-backends/src/wrapping/stark_to_groth16.rs:2324-2346).  `out` holds
 * 2^(log_h+log_blowup) x width elements.  shift = 0 selects the field generator. */
ZKB_API int zkb_coset_lde_batch(int field, const void *trace, uint32_t log_h, uint32_t width,
                        uint32_t log_blowup, uint64_t shift, int bitrev_rows, void *out);
ZKB_API int zkb_coset_lde_batch_dev(int field, const void *d_trace, uint32_t log_h, uint32_t width,
                            uint32_t log_blowup, uint64_t shift, int bitrev_rows, void *d_out,
                            void *stream);
/* The device LDE (generator shift, bit-reversed rows) with explicit kernel shapes:
 * largest NTT pass kmax index bits (1..11 BabyBear, 1..10 Goldilocks; 0 = default) and
 * the widest column chunk per CTA of the plain passes (1/4/8/16, 0 = default) and of the
 * fused middle kernel (1/4/8, 0 = default); columns beyond a multiple of the chunk take
 * narrower chunks.  Every choice gives the same output; the batched plan's
 * autotuner picks among them.  No counterpart in the reference (its Metal NTT has one
 * fixed dispatch shape, zkf-metal/src/ntt/p3_adapter.rs:78-294). */
ZKB_API int zkb_coset_lde_tuned_dev(int field, const void *d_trace, uint32_t log_h, uint32_t width,
                                    uint32_t log_blowup, int kmax, uint32_t c_pass, uint32_t c_fused,
                                    void *d_out, void *stream);

/* ------------------------------------------------------------------- MMCS */
/* A row-major matrix: `data` is a host or device pointer depending on the call. */
typedef struct {
  const void *data;
  uint64_t height;
  uint64_t width;
} zkb_matrix;

/* Poseidon2 hash configuration of an MMCS: PaddingFreeSponge<Perm, W, 8, OUT> leaves
 * and TruncatedPermutation<Perm, 2, OUT, W> nodes (zkf-backends/src/plonky3.rs:55-56),
 * Perm = Poseidon2 of `width` (16; Goldilocks also 12 with OUT = 4) with the
 * constants of `seed` (plonky3.rs:614-620, 1104-1111). */
typedef struct {
  int field;
  uint32_t width;
  uint64_t seed;
} zkb_hasher;

typedef struct zkb_tree zkb_tree;

/* Mmcs::commit (MetalMerkleTreeMmcs::commit, zkf-metal/src/merkle.rs:76-105;
 * p3 MerkleTree::new, vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:84-151), with no
 * width limit.  Matrices of several heights are allowed under p3's rule (heights
 * that round up to the same power of two are equal).  Host form: matrices are host
 * pointers and are copied to the device.  `root_out` receives OUT elements.
 * `tree_out` (may be NULL) receives the prover data, freed with zkb_tree_free. */
ZKB_API int zkb_mmcs_commit(const zkb_hasher *hasher, const zkb_matrix *mats, size_t n_mats,
                    void *root_out, zkb_tree **tree_out);
/* Device form: matrices are device pointers that must outlive the tree. */
ZKB_API int zkb_mmcs_commit_dev(const zkb_hasher *hasher, const zkb_matrix *d_mats, size_t n_mats,
                        void *root_out, zkb_tree **tree_out, void *stream);
/* Mmcs::commit of one device matrix (BabyBear, width-16 hasher) that also writes the
 * alpha-reduction of every row, d_codeword[i] = sum_j alpha^j * mat[i][j] over the quartic
 * extension (4 u32 per row, 16-byte aligned), in the same pass as the leaf hash — the
 * reduction zkb_combine_columns_babybear_ext4_dev computes separately.  For a caller that
 * knows alpha before the commitment (seeded challenges), e.g. one rank's row block of a
 * commitment split over GPUs. */
ZKB_API int zkb_mmcs_commit_reduce_dev(const zkb_hasher *hasher, const zkb_matrix *d_mat, const uint32_t *alpha,
                                       void *root_out, zkb_tree **tree_out, uint32_t *d_codeword, void *stream);
/* Digest layers (MerkleTree::digest_layers, merkle_tree.rs:40-54). */
ZKB_API int zkb_tree_num_layers(const zkb_tree *tree);
ZKB_API int64_t zkb_tree_layer_len(const zkb_tree *tree, int layer);
ZKB_API int zkb_tree_digest_elems(const zkb_tree *tree);
ZKB_API int zkb_tree_copy_layer(const zkb_tree *tree, int layer, void *host_out);
/* Mmcs::open_batch (vendor/p3-merkle-tree-gpu/src/mmcs.rs:179-210): rows of every
 * committed matrix at the reduced index, concatenated in commit order, and the
 * log2(max_height) sibling digests. */
ZKB_API int zkb_mmcs_open_batch(const zkb_tree *tree, uint64_t index, void *rows_out, size_t rows_cap,
                        void *siblings_out, size_t siblings_cap);
ZKB_API void zkb_tree_free(zkb_tree *tree);
/* Mmcs::verify_batch (vendor/p3-merkle-tree-gpu/src/mmcs.rs:230-330): checks one opening
 * against `root` (OUT elements).  heights/widths describe the committed matrices in
 * commit order; `rows` holds the opened row of every matrix, concatenated in commit
 * order; `siblings` holds n_siblings = log2(next_pow2(max height)) digests.  ZKB_OK when
 * the path reproduces the root; ZKB_ERR_INVALID (message: why) otherwise.  Elements are
 * u32 (BabyBear) or u64 (Goldilocks).  Host-side; needs no device. */
ZKB_API int zkb_mmcs_verify_batch(const zkb_hasher *hasher, const void *root, const uint64_t *heights,
                                  const uint64_t *widths, size_t n_mats, uint64_t index, const void *rows,
                                  const void *siblings, size_t n_siblings);

/* TruncatedPermutation<Perm, 2, OUT, W> (zkf-backends/src/plonky3.rs:56) of n digest pairs:
 * out[i] = compress(left[i], right[i]), OUT elements per digest (8 for width 16, 4 for
 * width 12), u32 (BabyBear) or u64 (Goldilocks).  It finishes the top levels of a tree
 * whose subtrees were built apart (one per device).  Host-side; needs no device. */
ZKB_API int zkb_mmcs_compress(const zkb_hasher *hasher, const void *left, const void *right, size_t n,
                              void *out);

/* TwoAdicFriPcs::commit for one trace matrix (the PCS type of
 * zkf-backends/src/plonky3.rs:68): coset LDE with shift = field generator, rows
 * bit-reversed, MMCS commit of the result — coset_lde_batch + bit_reverse_rows +
 * Mmcs::commit in one call.  The LDE (2^(log_h+log_blowup) x width) stays on the
 * device as the tree's leaf matrix, so openings read it without a copy.
 * Host form: `trace` is a host pointer (pinned memory gives full copy bandwidth).  A
 * BabyBear trace of 128 or more columns (width-16 hasher) crosses the link a 64-column slab
 * at a time, and each slab's LDE and leaf absorption run while the next slab is copied
 * (the same for zkb_pcs_commit_fri and engine jobs); results are the device form's. */
ZKB_API int zkb_pcs_commit(const zkb_hasher *hasher, const void *trace, uint32_t log_h,
                           uint32_t width, uint32_t log_blowup, void *root_out, zkb_tree **tree_out);
ZKB_API int zkb_pcs_commit_dev(const zkb_hasher *hasher, const void *d_trace, uint32_t log_h,
                               uint32_t width, uint32_t log_blowup, void *root_out,
                               zkb_tree **tree_out, void *stream);
/* Device pointer to the committed leaf matrix `mat` of a tree (for device-resident
 * follow-up work such as the FRI input); NULL on error. */
ZKB_API const void *zkb_tree_matrix_dev(const zkb_tree *tree, int mat);

/* ---------------------------------------------------------------------- FRI */
/* FriAccelerator::fold_goldilocks (zkf-core/src/acceleration.rs:197-217) and
 * MetalFri::fold_{goldilocks,babybear} (zkf-metal/src/fri.rs:36-147):
 *   out[i] = (e[2i] + e[2i+1]) / 2 + alpha * (e[2i] - e[2i+1]) * inv_twiddles[i].
 * n_evals is even; out holds n_evals/2 elements.  inv_twiddles = NULL selects
 * g^-rev(i)/2 with g = two_adic_generator(log2(n_evals)), which makes the fold
 * equal to p3 TwoAdicFriFolding::fold_matrix. */
ZKB_API int zkb_fri_fold_goldilocks(const uint64_t *evals, size_t n_evals, uint64_t alpha,
                            const uint64_t *inv_twiddles, uint64_t *out);
ZKB_API int zkb_fri_fold_babybear(const uint32_t *evals, size_t n_evals, uint32_t alpha,
                          const uint32_t *inv_twiddles, uint32_t *out);
/* p3 TwoAdicFriFolding::fold_matrix over the BabyBear quartic extension
 * (BinomialExtensionField<BabyBear, 4>, x^4 = 11): evals holds 2*n_out extension
 * elements (4 u32 each) in bit-reversed domain order; beta is 4 u32. */
ZKB_API int zkb_fri_fold_babybear_ext4(const uint32_t *evals, size_t n_out, const uint32_t *beta,
                               uint32_t *out);

/* FRI commit phase over the BabyBear quartic extension with seeded challenges — the
 * prove_fri commit phase and query answers of p3-fri 0.4.2 as TwoAdicFriPcs runs them
 * (PCS at zkf-backends/src/plonky3.rs:68, FRI parameters :597), folding with
 * p3 fold_matrix (see zkb_fri_fold_babybear_ext4).  Round r commits the codeword
 * (2^(log_n-r) extension elements, bit-reversed domain order) as rows of the pairs
 * (x, -x), 8 base elements each (ExtensionMmcs flattening), then folds with beta_r.
 * beta_r = four BabyBear draws (p3 sampler) from SmallRng(challenge_seed); query
 * indices are next_u64() >> (64 - log_n) from SmallRng(query_seed).  Each query opens,
 * per round, the row (index >> r) >> 1 and its sibling path.
 * With `transcript` set the challenges come from a DuplexChallenger over the BabyBear
 * width-16 Poseidon2 of the hasher (see zkb_challenger_*), as p3's prover draws them:
 * round r observes its root (8 elements) and samples beta_r (4 samples), the final
 * codeword is observed (element by element, 4 coefficients each), and every query
 * index is sample_bits(log_n).  The seeds are then unused.  The standalone FRI starts
 * from a fresh challenger; the commit+FRI job first observes the trace root and samples
 * alpha.  (p3 observes the final polynomial's coefficients; this transcript observes
 * the final codeword, which determines them.) */
typedef struct {
  uint32_t log_n;           /* codeword length 2^log_n extension elements */
  uint32_t log_final;       /* stop at 2^log_final elements */
  uint64_t challenge_seed;  /* betas (seeded mode) */
  uint32_t num_queries;
  uint64_t query_seed;      /* query indices (seeded mode) */
  uint32_t transcript;      /* 1: challenges from the Fiat-Shamir transcript */
} zkb_fri_params;
typedef struct zkb_fri_proof zkb_fri_proof;
/* Host form: `codeword` holds 2^log_n x 4 u32 (coefficients of each element). */
ZKB_API int zkb_fri_commit_babybear_ext4(const zkb_hasher *hasher, const zkb_fri_params *params,
                                         const uint32_t *codeword, zkb_fri_proof **proof_out);
ZKB_API int zkb_fri_commit_babybear_ext4_dev(const zkb_hasher *hasher, const zkb_fri_params *params,
                                             const uint32_t *d_codeword, zkb_fri_proof **proof_out,
                                             void *stream);
ZKB_API int zkb_fri_num_rounds(const zkb_fri_proof *proof);
/* Per-round commitments (rounds x 8 u32) and challenges (rounds x 4 u32). */
ZKB_API int zkb_fri_commitments(const zkb_fri_proof *proof, uint32_t *roots_out, uint32_t *betas_out);
/* Final codeword: 2^log_final x 4 u32. */
ZKB_API int zkb_fri_final_codeword(const zkb_fri_proof *proof, uint32_t *out);
/* Sibling elements per query (sum over rounds of (log_n - r - 1) x 8). */
ZKB_API int64_t zkb_fri_siblings_per_query(const zkb_fri_proof *proof);
/* Query answers: indices (num_queries), opened rows (num_queries x rounds x 8 u32) and
 * sibling paths (num_queries x siblings_per_query u32), round-major within a query. */
ZKB_API int zkb_fri_query_openings(const zkb_fri_proof *proof, uint64_t *indices_out,
                                   uint32_t *rows_out, uint32_t *siblings_out);
/* The alpha of the column reduction of a commit+FRI job: the caller's in seeded mode,
 * the transcript's in transcript mode (4 u32). */
ZKB_API int zkb_fri_alpha(const zkb_fri_proof *proof, uint32_t *alpha_out);
ZKB_API void zkb_fri_proof_free(zkb_fri_proof *proof);

/* ------------------------------------------------------------ transcript
 * p3's DuplexChallenger<F, Poseidon2<16>, 16, 8> (ZirOS: zkf-backends/src/plonky3.rs:66;
 * native restatement zkf-backends/src/wrapping/duplex_challenger.rs:1-145) over the
 * width-16 Poseidon2 of `hasher`.  Values are canonical field elements in u64.
 * sample_bits(b) = the next sample's low b bits (as stark_to_groth16.rs:2229-2255 uses
 * it).  Host-side; needs no device. */
typedef struct zkb_challenger zkb_challenger;
ZKB_API int zkb_challenger_create(const zkb_hasher *hasher, zkb_challenger **out);
ZKB_API int zkb_challenger_observe(zkb_challenger *c, const uint64_t *values, size_t n);
ZKB_API int zkb_challenger_sample(zkb_challenger *c, uint64_t *values_out, size_t n);
ZKB_API int zkb_challenger_sample_bits(zkb_challenger *c, uint32_t bits, uint64_t *out);
ZKB_API void zkb_challenger_free(zkb_challenger *c);
/* The FRI commit phase driven by a caller's transcript: like zkb_fri_commit_babybear_ext4_dev
 * in transcript mode (params->transcript and the seeds are ignored), but the challenger is
 * the caller's, in whatever state earlier observations left it, and it is advanced by the
 * call — as p3's prover threads one challenger from the trace commitment through alpha into
 * FRI (p3-fri 0.4.2 prove, over zkf-backends/src/plonky3.rs:66).  Used when the trace root is
 * known before the reduced codeword exists on this device (a commitment built over several
 * devices). */
ZKB_API int zkb_fri_commit_babybear_ext4_challenger_dev(const zkb_hasher *hasher,
                                                        const zkb_fri_params *params,
                                                        const uint32_t *d_codeword,
                                                        zkb_challenger *challenger,
                                                        zkb_fri_proof **proof_out, void *stream);

/* The batched codeword of a PCS opening, without the division by (x - z): for each LDE
 * row i, out[i] = sum_j alpha^j * lde[i][j] in the BabyBear quartic extension — the
 * alpha-reduction TwoAdicFriPcs applies to the committed columns before FRI
 * (p3-fri 0.4.2 open, PCS at zkf-backends/src/plonky3.rs:68).  Device pointers:
 * `d_lde` rows x width u32, `d_out` rows x 4 u32 (16-byte aligned). */
ZKB_API int zkb_combine_columns_babybear_ext4_dev(const uint32_t *d_lde, uint64_t rows, uint32_t width,
                                                  const uint32_t *alpha, uint32_t *d_out, void *stream);

/* One commitment job of the Plonky3 PCS for a BabyBear trace, device-resident from end
 * to end: zkb_pcs_commit (coset LDE, bit-reversed rows, MMCS), then the alpha-reduction
 * of the committed LDE columns into one F_p^4 codeword (zkb_combine_columns_...), then
 * the FRI commit phase and query answers on it (zkb_fri_commit_babybear_ext4;
 * params->log_n is set to log_h + log_blowup).  This is TwoAdicFriPcs commit + open
 * without the (x - z) quotient (PCS at zkf-backends/src/plonky3.rs:68).  With
 * params->transcript set, `alpha` is ignored: the transcript observes the trace root
 * and samples alpha, then drives the FRI challenges (zkb_fri_alpha returns it).
 * Outputs: the trace root (8 u32), the tree (may be NULL) and the FRI proof (may be NULL). */
ZKB_API int zkb_pcs_commit_fri(const zkb_hasher *hasher, const void *trace, uint32_t log_h,
                               uint32_t width, uint32_t log_blowup, const uint32_t *alpha,
                               const zkb_fri_params *params, void *root_out, zkb_tree **tree_out,
                               zkb_fri_proof **fri_out);
ZKB_API int zkb_pcs_commit_fri_dev(const zkb_hasher *hasher, const void *d_trace, uint32_t log_h,
                                   uint32_t width, uint32_t log_blowup, const uint32_t *alpha,
                                   const zkb_fri_params *params, void *root_out, zkb_tree **tree_out,
                                   zkb_fri_proof **fri_out, void *stream);

/* ------------------------------------------------------------ polynomial ops
 * PolyOpsAccelerator (zkf-core/src/acceleration.rs:173-194; Metal implementation
 * zkf-metal/src/poly.rs:37-230), Goldilocks, host pointers, canonical values:
 *   eval:       out[j] = f(points[j]) (Horner over n_coeffs coefficients, c_0 first);
 *   coset_eval: out[i] = f(shift * w^i), i < 2^log_n, for 2^log_n coefficients;
 *   quotient:   out[i] = (evals[i] - f_z) / (w^i - z) on the subgroup of size 2^log_n,
 *               0 where w^i = z. */
ZKB_API int zkb_poly_eval_goldilocks(const uint64_t *coeffs, size_t n_coeffs, const uint64_t *points,
                                     size_t n_points, uint64_t *out);
ZKB_API int zkb_poly_coset_eval_goldilocks(const uint64_t *coeffs, uint32_t log_n, uint64_t shift, uint64_t *out);
ZKB_API int zkb_poly_quotient_goldilocks(const uint64_t *evals, uint32_t log_n, uint64_t z, uint64_t f_z,
                                         uint64_t *out);

/* ---------------------------------------------------------------- runtime driver
 * A dispatch driver for the prover runtime's graph nodes (the reference's
 * GpuDispatchDriver, zkf-runtime/src/metal_driver.rs:55-80, over the ProverOp set of
 * zkf-runtime/src/graph.rs:51-110): device buffer slots, and nodes that read and write
 * them, each depending only on earlier nodes, executed in order on one stream.  A node
 * the device path declines (thresholds, kill switch, open circuit) stops the run with
 * ZKB_DECLINED and names the node in *fallback_node (the reference's FallbackSignal: the
 * caller runs that node and the rest on the CPU).  Sizes: rows = 2^log_n. */
#define ZKB_OP_NTT 1              /* in place on in_slot: rows x width, natural order; inverse */
#define ZKB_OP_LDE 2              /* in_slot rows x width -> out_slot (rows << log_blowup) x width, bit-reversed rows */
#define ZKB_OP_POSEIDON_BATCH 3   /* in place on in_slot: count width-16 states; seed */
#define ZKB_OP_MERKLE 4           /* MMCS of in_slot (rows x width); root -> out_slot (may be -1); seed, hasher_width */
#define ZKB_OP_FRI_FOLD 5         /* in_slot 2^log_n evaluations -> out_slot 2^(log_n-1); beta; ext4: F_p^4 BabyBear */
#define ZKB_OP_FRI_QUERY_OPEN 6   /* tree of node tree_node at count u64 indices (in_slot) -> out_slot: per query the
                                     row then its sibling digests */
typedef struct {
  int kind;                /* ZKB_OP_* */
  int field;               /* ZKB_FIELD_* */
  uint32_t log_n, width, log_blowup, inverse;
  uint64_t count;
  int in_slot, out_slot;
  uint64_t seed;           /* Poseidon2 seed (PoseidonBatch, Merkle) */
  uint32_t hasher_width;   /* Merkle: 16 (default when 0) or 12 (Goldilocks) */
  uint32_t ext4;           /* FriFold over BabyBear^4 */
  uint32_t beta[4];        /* FriFold challenge (base field: beta[0], or beta[1]:beta[0] for Goldilocks) */
  int tree_node;           /* FriQueryOpen: the Merkle node whose tree is opened */
} zkb_rt_node;
typedef struct zkb_rt zkb_rt;
ZKB_API int zkb_rt_create(zkb_rt **rt_out);
ZKB_API int zkb_rt_buffer(zkb_rt *rt, uint64_t bytes, int *slot_out);
ZKB_API int zkb_rt_write(zkb_rt *rt, int slot, const void *host, uint64_t bytes);
ZKB_API int zkb_rt_read(zkb_rt *rt, int slot, void *host, uint64_t bytes);
ZKB_API int zkb_rt_add(zkb_rt *rt, const zkb_rt_node *node, const int *deps, size_t n_deps, int *node_id);
ZKB_API int zkb_rt_execute(zkb_rt *rt, void *stream, int *fallback_node);
/* Device time of a node in the last successful run (CUDA events around its launches). */
ZKB_API int zkb_rt_node_ms(const zkb_rt *rt, int node_id, float *ms);
/* Tree of an executed Merkle node (borrowed; zkb_mmcs_open_batch works on it). */
ZKB_API int zkb_rt_tree(const zkb_rt *rt, int node_id, const zkb_tree **tree);
ZKB_API void zkb_rt_free(zkb_rt *rt);

/* ---------------------------------------------------------------- serving */
/* Continuous-batching engine for commit jobs (the role of the reference's proof-level
 * scheduler, zkf-metal/src/batch_prover.rs:94-140, and its bounded in-flight pipeline,
 * zkf-metal/src/pipeline.rs:23-126).  `slots` worker threads each own a stream; a
 * queued job is admitted when its device-memory estimate fits the HBM budget (in the
 * order `policy` gives), runs with its LDE, trees and FRI layers
 * device-resident, and releases its memory when its answers are on the host.  Jobs on
 * different slots overlap on the GPU; a job's results depend only on its inputs. */
typedef struct {
  uint32_t slots;        /* concurrent jobs */
  uint64_t hbm_budget;   /* bytes for job state; 0 = free device memory minus 2 GiB */
  uint32_t policy;       /* admission: ZKB_ADMIT_FIFO (0, the default) or ZKB_ADMIT_SMALLEST */
} zkb_engine_config;
/* FIFO: the oldest queued job that fits the remaining budget (a job waiting for memory may
 * be passed by younger jobs that fit).  SMALLEST: the fitting job with the fewest trace
 * cells.  Under both, a job passed over ZKB_ADMIT_MAX_BYPASS times is admitted next, and
 * while it does not fit nothing else is admitted (no job waits forever).  Whatever the
 * policy, a running job's stream priority follows its size (small jobs' kernels are
 * scheduled first as blocks retire), trace uploads take the link piece by piece with the
 * fewest bytes left first, and one job per size class runs its LDE and tree at a time. */
#define ZKB_ADMIT_FIFO 0
#define ZKB_ADMIT_SMALLEST 1
#define ZKB_ADMIT_MAX_BYPASS 8
typedef struct {
  zkb_hasher hasher;
  const void *trace;     /* host memory (pinned for full copy bandwidth), valid until done */
  uint32_t log_h, width, log_blowup;
  int with_fri;          /* BabyBear: alpha-reduction + FRI commit phase after the commit */
  uint32_t alpha[4];
  zkb_fri_params fri;    /* log_n is set from the trace */
} zkb_job_desc;
typedef struct {
  int status;            /* ZKB_OK or the job's error */
  uint32_t root[16];     /* OUT elements (u32 BabyBear; Goldilocks digests as 2 u32 each) */
  double queue_ms, run_ms, latency_ms;
} zkb_job_result;
typedef struct {
  uint64_t queued, completed, hbm_budget, hbm_in_use, hbm_peak;
} zkb_engine_stats_t;
typedef struct zkb_engine zkb_engine;
ZKB_API int zkb_engine_create(const zkb_engine_config *config, zkb_engine **engine_out);
/* Non-blocking; the descriptor is copied. */
ZKB_API int zkb_engine_submit(zkb_engine *engine, const zkb_job_desc *job, uint64_t *job_id);
/* Blocks until the job is done; fri_out (may be NULL) receives its FRI answers. */
ZKB_API int zkb_engine_wait(zkb_engine *engine, uint64_t job_id, zkb_job_result *result,
                            zkb_fri_proof **fri_out);
/* Cancels a job that is still queued (its wait then returns ZKB_ERR_CANCELLED);
 * ZKB_DECLINED when it has already started. */
ZKB_API int zkb_engine_cancel(zkb_engine *engine, uint64_t job_id);
ZKB_API int zkb_engine_stats(zkb_engine *engine, zkb_engine_stats_t *stats);
/* Finishes the queued jobs, then stops the workers. */
ZKB_API void zkb_engine_destroy(zkb_engine *engine);

/* ------------------------------------------------------------------ batched commit
 * Many traces of uneven height and width committed by one plan.  Replaces a loop of
 * per-trace commits (TwoAdicFriPcs::commit over one matrix each,
 * zkf-metal/src/merkle.rs:55-138 with the LDE of zkf-metal/src/ntt/p3_adapter.rs:78-294);
 * every root equals that trace's plain commitment (zkb_pcs_commit).
 * zkb_batch_create allocates every device buffer once, builds the tables, picks the
 * kernel shapes (timed candidates when `autotune`, cached as JSON lines in
 * `tune_cache`) and captures one CUDA graph; zkb_batch_run replays it.  A plan is
 * used by one thread at a time; runs on different streams must not overlap. */
typedef struct {
  uint32_t log_h;        /* trace height 2^log_h */
  uint32_t width;        /* columns, 1..4096 */
} zkb_batch_shape;
typedef struct {
  uint32_t log_blowup;   /* 1..4 */
  int use_graph;         /* 1: one CUDA graph per run; 0: the same launches on streams;
                            2: one persistent kernel per run, fed by a device work queue and
                            captured in a CUDA graph (BabyBear, width-16 hasher, widths that
                            are multiples of 8, 2^(log_h + log_blowup) <= 2^25) */
  uint32_t branches;     /* concurrent LDE branches (1..8); 0 = tuned/default */
  int autotune;          /* time kernel-shape candidates at creation */
  const char *tune_cache;/* JSON-lines file read (and rewritten after tuning); NULL = none */
} zkb_batch_options;
typedef struct {
  uint64_t device_bytes; /* the plan's arena */
  uint32_t kernels_per_run; /* kernel nodes of the graph (0 without a graph) */
  uint32_t branches;
  uint32_t leaf_threads;
  int use_graph;
  int tuned_from_cache;
  double tune_ms;        /* device time spent building tables and tuning */
} zkb_batch_info_t;
typedef struct zkb_batch zkb_batch;
ZKB_API int zkb_batch_create(const zkb_hasher *hasher, const zkb_batch_shape *shapes, size_t n,
                             const zkb_batch_options *options, zkb_batch **batch_out);
/* Device buffer of trace i (2^log_h x width, row-major), for callers that write it in place. */
ZKB_API int zkb_batch_trace_ptr(zkb_batch *batch, size_t i, void **d_trace);
/* Copies trace i in from host (pinned for full bandwidth) or device memory. */
ZKB_API int zkb_batch_copy_in(zkb_batch *batch, size_t i, const void *src, int src_on_device, void *stream);
ZKB_API int zkb_batch_run(zkb_batch *batch, void *stream);
/* One run whose traces come from host memory: traces[i] points to trace i (2^log_h x width,
 * row-major, canonical elements; pinned host memory for the copies to run asynchronously).
 * The copies overlap the commitment: a copy stream takes the traces in groups (about 1/64
 * of the batch's cells each, small traces first and last, the largest in the middle), and
 * each group's LDEs and trees — one graph per group, captured at the plan's first host run
 * (which also allocates the second lane below) — run as soon as
 * the group's copies have landed, the groups alternating between `stream` and a second
 * stream of the plan (with a second coefficient-scratch set, when it takes at most 1/8 of
 * free device memory); `stream` waits for all of it.  A persistent plan copies every trace first,
 * then runs its kernel.  Pinned sources are read until
 * `stream` has passed the run; pageable ones are staged before the call returns.  Roots
 * and trees as after zkb_batch_run.  No counterpart in the reference. */
ZKB_API int zkb_batch_run_host(zkb_batch *batch, const void *const *traces, void *stream);
/* n x OUT root elements (Goldilocks digests as u64); synchronises `stream`. */
ZKB_API int zkb_batch_roots(zkb_batch *batch, void *roots_out, void *stream);
/* Borrowed tree of trace i (valid while the plan lives, contents after a finished run):
 * zkb_mmcs_open_batch and the zkb_tree_* accessors work on it; do not free it. */
ZKB_API int zkb_batch_tree(zkb_batch *batch, size_t i, const zkb_tree **tree);
ZKB_API int zkb_batch_info(const zkb_batch *batch, zkb_batch_info_t *info);
/* Kernel shapes chosen for trace i's LDE (0 = default). */
ZKB_API int zkb_batch_lde_tune(const zkb_batch *batch, size_t i, int *kmax, uint32_t *c_pass,
                               uint32_t *c_fused);
/* Merkle-level fusion of a persistent plan (use_graph = 2): the levels above the leaves
 * that each leaf-hash tile of 256 rows also computes in shared memory (0..8), and the
 * levels each compression tile computes (1..8).  Rebuilds the work queue and the graph;
 * the autotuner sets them at creation.  No counterpart in the reference. */
ZKB_API int zkb_batch_set_merkle_fusion(zkb_batch *batch, uint32_t leaf_levels, uint32_t comp_levels);
typedef struct {
  uint32_t items;        /* work items in the queue */
  uint32_t steps;        /* dependency steps (one counter each) */
  uint32_t stages;
  uint32_t grid;         /* blocks of the persistent kernel */
  uint32_t leaf_levels, comp_levels;
} zkb_batch_queue_info_t;
ZKB_API int zkb_batch_queue_info(const zkb_batch *batch, zkb_batch_queue_info_t *info);
/* One profiled run of a persistent plan (waits for it): busy_ms[4] = the blocks' summed
 * busy time on NTT passes, fused LDE middles, leaf hashing and compression items; span_ms
 * = first item start to last item end (global timer).  No counterpart in the reference. */
ZKB_API int zkb_batch_profile(zkb_batch *batch, void *stream, double *busy_ms, double *span_ms);
/* Test hook of a persistent plan: one run (not the graph) in which a work item waits on a
 * counter that nothing bumps, polling at most spin_limit times (1..2^24) before it gives up;
 * the kernel then records the item, every block leaves the queue, and the next
 * zkb_batch_roots returns ZKB_ERR_TIMEOUT.  The run's results are invalid; the next
 * zkb_batch_run recomputes everything.  No device fault is involved. */
ZKB_API int zkb_debug_batch_stalled_run(zkb_batch *batch, uint64_t spin_limit, void *stream);
ZKB_API void zkb_batch_free(zkb_batch *batch);

#ifdef __cplusplus
}
#endif
#endif /* ZKB200_H */
