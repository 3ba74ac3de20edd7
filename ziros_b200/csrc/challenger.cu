// challenger.cu — the Fiat-Shamir transcript of the FRI prover.
//
// DuplexChallenger<F, Poseidon2<16>, 16, 8> (p3-challenger 0.4.2 as ZirOS uses it,
// zkf-backends/src/plonky3.rs:66; restated natively in
// zkf-backends/src/wrapping/duplex_challenger.rs:1-145):
//   observe(x):  clears the output buffer, appends x to the input buffer and duplexes
//                when the input buffer holds RATE = 8 elements;
//   sample():    duplexes when there is pending input or no output left, then pops the
//                LAST element of the output buffer;
//   duplexing:   overwrites state[0..len(input)] with the input (the rest of the rate
//                is kept), permutes, and refills the output buffer with state[0..8];
//   sample_bits(b): sample() as a canonical integer, masked to its low b bits
//                (stark_to_groth16.rs:2229-2255 uses it for PoW checks and query indices).
// An F_p^4 challenge is four samples, coefficient 0 first.  It runs on the host: a few
// permutations per FRI round, with the permutation code the kernels use.
#include <cstring>
#include <memory>

#include "common.cuh"
#include "engine.cuh"

namespace zkb {

int DuplexChallenger::init(const HasherSpec &s) {
  ZKB_REQUIRE(s.width == 16, "the challenger permutes width-16 states");
  spec = s;
  std::memset(state, 0, sizeof state);
  in.clear();
  out.clear();
  const bool ok = s.field == FIELD_BABYBEAR ? build_p2_params<BabyBear, 16>(s, &p_bb)
                                            : build_p2_params<Goldilocks, 16>(s, &p_gl);
  ZKB_REQUIRE(ok, "invalid Poseidon2 parameters");
  return ZKB_OK;
}

void DuplexChallenger::permute() {
  if (spec.field == FIELD_BABYBEAR) {
    uint32_t s[16];
    for (int i = 0; i < 16; i++) s[i] = Dom<BabyBear>::enter((uint32_t)state[i]);
    p2_permute<BabyBear, 16>(s, p_bb);
    for (int i = 0; i < 16; i++) state[i] = Dom<BabyBear>::leave(s[i]);
  } else {
    uint64_t s[16];
    for (int i = 0; i < 16; i++) s[i] = state[i];
    p2_permute<Goldilocks, 16>(s, p_gl);
    for (int i = 0; i < 16; i++) state[i] = s[i];
  }
}

void DuplexChallenger::duplexing() {
  for (size_t i = 0; i < in.size(); i++) state[i] = in[i];
  in.clear();
  permute();
  out.assign(state, state + 8);
}

void DuplexChallenger::observe(uint64_t v) {
  out.clear();
  in.push_back(v);
  if (in.size() == 8) duplexing();
}

uint64_t DuplexChallenger::sample() {
  if (!in.empty() || out.empty()) duplexing();
  const uint64_t v = out.back();
  out.pop_back();
  return v;
}

uint64_t DuplexChallenger::sample_bits(int bits) {
  const uint64_t v = sample();
  return bits >= 64 ? v : (v & ((1ull << bits) - 1));
}

}  // namespace zkb

using namespace zkb;

extern "C" {

int zkb_challenger_create(const zkb_hasher *hasher, zkb_challenger **out) {
  clear_error();
  ZKB_REQUIRE(hasher && out, "null arguments");
  HasherSpec spec;
  if (!make_hasher_spec(hasher->field, (int)hasher->width, hasher->seed, &spec)) {
    set_error("unsupported Poseidon2 hasher: field %d width %u", hasher->field, hasher->width);
    return ZKB_ERR_UNSUPPORTED;
  }
  auto c = std::make_unique<zkb_challenger>();
  ZKB_TRY(c->c.init(spec));
  *out = c.release();
  return ZKB_OK;
}

int zkb_challenger_observe(zkb_challenger *c, const uint64_t *values, size_t n) {
  clear_error();
  ZKB_REQUIRE(c && (values || n == 0), "null arguments");
  const uint64_t p = c->c.spec.field == FIELD_BABYBEAR ? BabyBear::P : Goldilocks::P;
  for (size_t i = 0; i < n; i++) ZKB_REQUIRE(values[i] < p, "observed value %zu is not canonical", i);
  for (size_t i = 0; i < n; i++) c->c.observe(values[i]);
  return ZKB_OK;
}

int zkb_challenger_sample(zkb_challenger *c, uint64_t *values_out, size_t n) {
  clear_error();
  ZKB_REQUIRE(c && (values_out || n == 0), "null arguments");
  for (size_t i = 0; i < n; i++) values_out[i] = c->c.sample();
  return ZKB_OK;
}

int zkb_challenger_sample_bits(zkb_challenger *c, uint32_t bits, uint64_t *out) {
  clear_error();
  ZKB_REQUIRE(c && out && bits <= 64, "invalid arguments");
  *out = c->c.sample_bits((int)bits);
  return ZKB_OK;
}

void zkb_challenger_free(zkb_challenger *c) { delete c; }

}  // extern "C"
