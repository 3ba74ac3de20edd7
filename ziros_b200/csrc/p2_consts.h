// p2_consts.h — Poseidon2 instance parameters on the host.
//
// Constants follow the reference's flatten_round_constants(seed)
// (zkf-metal/src/poseidon2/babybear.rs:76-111, goldilocks.rs:42-83): rand 0.9
// SmallRng::seed_from_u64(seed) (xoshiro256++ expanded by SplitMix64), then
// ExternalLayerConstants::new_from_rng(R_F) (R_F/2 initial then R_F/2 terminal
// width-arrays) and R_P internal draws.  Flat layout [initial | internal | terminal].
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace zkb {

enum FieldId : int { FIELD_BABYBEAR = 0, FIELD_GOLDILOCKS = 1 };

struct SmallRng {
  uint64_t s[4];
  explicit SmallRng(uint64_t seed);
  uint64_t next_u64();
  uint32_t next_u32() { return (uint32_t)(next_u64() >> 32); }
};

// Canonical draws matching p3's StandardUniform samplers.
uint64_t sample_goldilocks(SmallRng &r);
uint32_t sample_babybear(SmallRng &r);  // 31-bit draw taken as Montgomery form

// poseidon2_round_numbers_128 (D = 7).  Returns false when unsupported.
bool p2_round_numbers(int field, int width, int *rounds_f, int *rounds_p);

// Canonical flat constants; empty on unsupported configuration.
std::vector<uint64_t> p2_flat_constants(int field, int width, uint64_t seed);
// Canonical internal diagonal (BabyBear W16 V, Goldilocks W16 MATRIX_DIAG_16, the
// self-generated Goldilocks W12 one).  Empty on unsupported configuration.
std::vector<uint64_t> p2_diagonal(int field, int width);

// A fully described Poseidon2 hash configuration: permutation + sponge geometry
// (PaddingFreeSponge<Perm, W, 8, OUT>, TruncatedPermutation<Perm, 2, OUT, W>).
struct HasherSpec {
  int field = 0;
  int width = 16;
  int rate = 8;
  int out = 8;
  int rounds_f = 0, rounds_p = 0;
  std::vector<uint64_t> rc;    // canonical
  std::vector<uint64_t> diag;  // canonical
};
bool make_hasher_spec(int field, int width, uint64_t seed, HasherSpec *out);

}  // namespace zkb
