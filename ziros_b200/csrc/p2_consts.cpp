// p2_consts.cpp — host generation of Poseidon2 constants (see p2_consts.h).
#include "p2_consts.h"

#include "field.cuh"

namespace zkb {

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

// SplitMix64 expansion of a u64 seed into the xoshiro256++ state.
SmallRng::SmallRng(uint64_t seed) {
  uint64_t state = seed;
  for (int i = 0; i < 4; i++) {
    state += 0x9e3779b97f4a7c15ull;
    uint64_t z = state;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    s[i] = z ^ (z >> 31);
  }
}

// xoshiro256++ (Blackman & Vigna).
uint64_t SmallRng::next_u64() {
  uint64_t res = rotl(s[0] + s[3], 23) + s[0];
  uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return res;
}

uint64_t sample_goldilocks(SmallRng &r) {
  for (;;) {
    uint64_t v = r.next_u64();
    if (v < Goldilocks::P) return v;
  }
}

uint32_t sample_babybear(SmallRng &r) {
  for (;;) {
    uint32_t v = r.next_u32() >> 1;
    if (v < BabyBear::P) return BabyBear::from_mont(v);
  }
}

bool p2_round_numbers(int field, int width, int *rf, int *rp) {
  if (field == FIELD_BABYBEAR) {
    if (width == 16) { *rf = 8; *rp = 13; return true; }
    if (width == 24) { *rf = 8; *rp = 21; return true; }
    return false;
  }
  if (field == FIELD_GOLDILOCKS && (width == 8 || width == 12 || width == 16 || width == 20)) {
    *rf = 8;
    *rp = 22;
    return true;
  }
  return false;
}

std::vector<uint64_t> p2_flat_constants(int field, int width, uint64_t seed) {
  int rf, rp;
  if (!p2_round_numbers(field, width, &rf, &rp)) return {};
  SmallRng r(seed);
  auto draw = [&]() -> uint64_t {
    return field == FIELD_BABYBEAR ? (uint64_t)sample_babybear(r) : sample_goldilocks(r);
  };
  std::vector<uint64_t> ext((size_t)rf * width);
  for (auto &v : ext) v = draw();
  std::vector<uint64_t> flat;
  size_t half = (size_t)(rf / 2) * width;
  flat.insert(flat.end(), ext.begin(), ext.begin() + half);
  for (int i = 0; i < rp; i++) flat.push_back(draw());
  flat.insert(flat.end(), ext.begin() + half, ext.end());
  return flat;
}

std::vector<uint64_t> p2_diagonal(int field, int width) {
  if (field == FIELD_BABYBEAR && width == 16) {
    // V = [-2, 1, 2, 1/2, 3, 4, -1/2, -3, -4, 1/2^8, 1/4, 1/8, 1/2^27, -1/2^8, -1/16, -1/2^27]
    // (zkf-metal/src/poseidon2/babybear.rs:14-58)
    const uint32_t P = BabyBear::P;
    uint32_t inv2 = inv_host<BabyBear>(2);
    auto ip = [&](int e) { return pow_host<BabyBear>(inv2, e); };
    return {P - 2, 1, 2, inv2, 3, 4, P - inv2, P - 3, P - 4, ip(8), ip(2), ip(3), ip(27),
            P - ip(8), P - ip(4), P - ip(27)};
  }
  if (field == FIELD_GOLDILOCKS && width == 16) {
    // MATRIX_DIAG_16_GOLDILOCKS (zkf-metal/src/poseidon2/goldilocks.rs:21-38)
    return {0xde9b91a467d6afc0ull, 0xc5f16b9c76a9be17ull, 0x0ab0fef2d540ac55ull,
            0x3001d27009d05773ull, 0xed23b1f906d3d9ebull, 0x5ce73743cba97054ull,
            0x1c3bab944af4ba24ull, 0x2faa105854dbafaeull, 0x53ffb3ae6d421a10ull,
            0xbcda9df8884ba396ull, 0xfc1273e4a31807bbull, 0xc77952573d5142c0ull,
            0x56683339a819b85eull, 0x328fcbd8f0ddc8ebull, 0xb5101e303fce9cb7ull,
            0x774487b8c40089bbull};
  }
  if (field == FIELD_GOLDILOCKS && width == 12) {
    // The reference ships no width-12 instance.  This diagonal is self-generated:
    // twelve distinct Goldilocks draws, each > 1, from SmallRng seeded with the ASCII
    // bytes "W12DIAG".  It is a parity-unpinned stand-in, not p3's constant.
    SmallRng r(0x57313244494147ull);
    std::vector<uint64_t> d;
    while (d.size() < 12) {
      uint64_t v = sample_goldilocks(r);
      bool ok = v > 1;
      for (uint64_t x : d) ok = ok && x != v;
      if (ok) d.push_back(v);
    }
    return d;
  }
  return {};
}

bool make_hasher_spec(int field, int width, uint64_t seed, HasherSpec *out) {
  HasherSpec h;
  h.field = field;
  h.width = width;
  h.rate = 8;
  h.out = width == 16 ? 8 : (width == 12 ? 4 : 0);
  if (!h.out) return false;
  if (!p2_round_numbers(field, width, &h.rounds_f, &h.rounds_p)) return false;
  h.rc = p2_flat_constants(field, width, seed);
  h.diag = p2_diagonal(field, width);
  if (h.rc.empty() || h.diag.empty()) return false;
  *out = std::move(h);
  return true;
}

}  // namespace zkb
