// poseidon2.cu — batch Poseidon2 permutation (Poseidon2Accelerator::batch_permute_*).
#include "common.cuh"
#include "engine.cuh"
#include "poseidon2.cuh"

namespace zkb {

template <class F, int W>
bool build_p2_params(const uint64_t *rc, size_t n_rc, int rounds_f, int rounds_p,
                     const uint64_t *diag, int out, P2Params<F, W> *p) {
  if (rounds_f <= 0 || rounds_f % 2 || rounds_p < 0) return false;
  if ((size_t)rounds_f * W + rounds_p != n_rc || n_rc > (size_t)P2_MAX_RC) return false;
  for (size_t i = 0; i < n_rc; i++) {
    if (rc[i] >= (uint64_t)F::P) return false;
    p->rc[i] = Dom<F>::encode(rc[i]);
  }
  for (int i = 0; i < W; i++) {
    if (diag[i] >= (uint64_t)F::P) return false;
    p->diag[i] = Dom<F>::encode(diag[i]);
  }
  p->rounds_f = rounds_f;
  p->rounds_p = rounds_p;
  p->out = out;
  p->rate = 8;
  p->diag_kind = 0;
  if (sizeof(typename F::T) == 4 && W == 16) {
    std::vector<uint64_t> v = p2_diagonal(FIELD_BABYBEAR, 16);
    bool same = true;
    for (int i = 0; i < W; i++) same = same && diag[i] == v[i];
    p->diag_kind = same ? 1 : 0;
  }
  return true;
}

template <class F, int W>
bool build_p2_params(const HasherSpec &h, P2Params<F, W> *p) {
  if (h.width != W) return false;
  return build_p2_params<F, W>(h.rc.data(), h.rc.size(), h.rounds_f, h.rounds_p, h.diag.data(),
                               h.out, p);
}

template <class F, int W>
__global__ void __launch_bounds__(128)
    p2_batch_kernel(typename F::T *__restrict__ states, size_t n,
                    const __grid_constant__ P2Params<F, W> p) {
  using T = typename F::T;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    T s[W];
    T *g = states + i * W;
#pragma unroll
    for (int k = 0; k < W; k++) s[k] = Dom<F>::enter(g[k]);
    p2_permute<F, W>(s, p);
#pragma unroll
    for (int k = 0; k < W; k++) g[k] = Dom<F>::leave(s[k]);
  }
}

template <class F, int W>
int p2_permute_batch(typename F::T *d_states, size_t n_states, const P2Params<F, W> &p,
                     cudaStream_t s) {
  if (n_states == 0) return ZKB_OK;
  DeviceContext *ctx;
  ZKB_TRY(current_context(&ctx));
  const unsigned threads = 128;
  unsigned grid = grid_for(n_states, threads, (unsigned)ctx->sm_count * 16u);
  ZKB_LAUNCH("p2_permute", s, p2_batch_kernel<F, W><<<grid, threads, 0, s>>>(d_states, n_states, p));
  ZKB_CHECK_LAUNCH();
  return ZKB_OK;
}

template bool build_p2_params<BabyBear, 16>(const uint64_t *, size_t, int, int, const uint64_t *,
                                            int, P2Params<BabyBear, 16> *);
template bool build_p2_params<Goldilocks, 16>(const uint64_t *, size_t, int, int,
                                              const uint64_t *, int, P2Params<Goldilocks, 16> *);
template bool build_p2_params<Goldilocks, 12>(const uint64_t *, size_t, int, int,
                                              const uint64_t *, int, P2Params<Goldilocks, 12> *);
template bool build_p2_params<BabyBear, 16>(const HasherSpec &, P2Params<BabyBear, 16> *);
template bool build_p2_params<Goldilocks, 16>(const HasherSpec &, P2Params<Goldilocks, 16> *);
template bool build_p2_params<Goldilocks, 12>(const HasherSpec &, P2Params<Goldilocks, 12> *);
template int p2_permute_batch<BabyBear, 16>(uint32_t *, size_t, const P2Params<BabyBear, 16> &,
                                            cudaStream_t);
template int p2_permute_batch<Goldilocks, 16>(uint64_t *, size_t,
                                              const P2Params<Goldilocks, 16> &, cudaStream_t);
template int p2_permute_batch<Goldilocks, 12>(uint64_t *, size_t,
                                              const P2Params<Goldilocks, 12> &, cudaStream_t);

}  // namespace zkb
