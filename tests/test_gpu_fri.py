"""FRI folding on the GPU vs the oracle (bit-exact).

Mirrors zkf-metal/src/fri.rs:200-224 (Goldilocks, 2048 outputs, evals 7i+1,
inverse twiddles 13i+3, alpha 42) and checks the p3 fold_matrix forms (base field
with computed twiddles, BabyBear quartic extension)."""
import numpy as np
import pytest

import ziros_b200 as Z
from conftest import GL_P, rand_field

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fri():
    f = Z.CudaFri.new()
    assert f is not None
    return f


def test_reference_fixture_goldilocks(oracle, fri):
    n = 2048
    ev = np.array([(i * 7 + 1) % GL_P for i in range(2 * n)], np.uint64)
    tw = np.array([(i * 13 + 3) % GL_P for i in range(n)], np.uint64)
    got = fri.fold_goldilocks(ev, 42, tw)
    assert got is not None and (got == oracle.fri_fold_base(1, ev, 42, tw)).all()


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("log_n", [0, 1, 5, 12, 18])
def test_fold_given_and_p3_twiddles(oracle, fri, field, log_n):
    n = 1 << log_n
    ev = rand_field(field, 2 * n, log_n)
    alpha = int(rand_field(field, 1, 99 + log_n)[0])
    tw = rand_field(field, n, 7 + log_n)
    fold = fri.fold_babybear if field == Z.BABYBEAR else fri.fold_goldilocks
    assert (fold(ev, alpha, tw) == oracle.fri_fold_base(field, ev, alpha, tw)).all()
    p3_tw = oracle.fri_inv_twiddles(field, n)
    assert (fold(ev, alpha) == oracle.fri_fold_base(field, ev, alpha, p3_tw)).all()


def test_fold_declines_bad_shapes(fri):
    assert fri.fold_goldilocks(np.zeros(5, np.uint64), 1, np.zeros(2, np.uint64)) is None
    assert fri.fold_goldilocks(np.zeros(8, np.uint64), 1, np.zeros(3, np.uint64)) is None


@pytest.mark.parametrize("log_n", [0, 3, 12, 20])
def test_fold_ext4_matches_oracle(oracle, fri, log_n):
    n = 1 << log_n
    ev = rand_field(Z.BABYBEAR, (2 * n, 4), 40 + log_n)
    beta = rand_field(Z.BABYBEAR, 4, 41 + log_n)
    assert (fri.fold_babybear_ext4(ev, beta) == oracle.fri_fold_ext4(ev, beta)).all()


def _check_fri(oracle, cw, log_final, nq, p2_seed=42, cseed=7, qseed=11):
    prover = Z.CudaFriProver(p2_seed, log_final, nq, cseed, qseed)
    pf = prover.commit(cw)
    want = oracle.fri_commit_ext4(cw, log_final, p2_seed, cseed, nq, qseed)
    assert (pf.betas == want["betas"]).all()
    assert (pf.roots == want["roots"]).all()
    assert (pf.final == want["final"]).all()
    assert (pf.query_indices == want["indices"]).all()
    for q in range(nq):
        for r in range(pf.rounds):
            row, proof = want["queries"][q][r]
            assert (pf.query_rows[q, r] == row).all()
            assert (pf.siblings(q, r) == np.array(proof).reshape(-1, 8)).all()
    return pf


@pytest.mark.parametrize("log_n,log_final,nq", [(1, 0, 3), (6, 2, 10), (12, 4, 20)])
def test_fri_commit_phase_matches_oracle(oracle, log_n, log_final, nq):
    cw = rand_field(Z.BABYBEAR, (1 << log_n, 4), 300 + log_n)
    _check_fri(oracle, cw, log_final, nq)


def test_fri_config3_full_size(oracle):
    """BabyBear F_p^4 codeword of 2^22 evaluations folded by 2 down to 2^8, every layer
    committed, 100 seeded queries: every root, layer path and fold output bit-exact."""
    cw = rand_field(Z.BABYBEAR, (1 << 22, 4), 2222)
    pf = _check_fri(oracle, cw, 8, 100)
    assert pf.rounds == 14 and pf.final.shape == (256, 4)


def test_fri_commit_device_resident(oracle):
    import torch

    cw = rand_field(Z.BABYBEAR, (1 << 10, 4), 5)
    t = torch.from_numpy(cw.view(np.int32)).cuda()
    pf = Z.CudaFriProver(3, 2, 5, 9, 13).commit_dev(t)
    want = oracle.fri_commit_ext4(cw, 2, 3, 9, 5, 13)
    assert (pf.roots == want["roots"]).all() and (pf.final == want["final"]).all()


@pytest.mark.parametrize("rows,width", [(1, 1), (64, 7), (1 << 12, 256), (100, 12), (33, 132), (40, 130)])
def test_combine_columns_matches_oracle(oracle, rows, width):
    import torch

    lde = rand_field(Z.BABYBEAR, (rows, width), rows + width)
    alpha = rand_field(Z.BABYBEAR, 4, 77)
    t = torch.from_numpy(lde.view(np.int32)).cuda()
    out = torch.zeros((rows, 4), dtype=torch.int32, device="cuda")
    Z.combine_columns_dev(t, alpha, out)
    torch.cuda.synchronize()
    assert (out.cpu().numpy().view(np.uint32) == oracle.combine_columns_ext4(lde, alpha)).all()


def test_pcs_commit_fri_job_matches_oracle(oracle):
    """One commitment job: LDE + MMCS of the trace, alpha-reduction of the LDE columns,
    FRI commit phase with queries — compared piece by piece with the oracle."""
    trace = rand_field(Z.BABYBEAR, (1 << 10, 24), 31)
    alpha = rand_field(Z.BABYBEAR, 4, 32)
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    root, tree, pf = pcs.commit_fri(trace, alpha, log_final=3, num_queries=10, challenge_seed=5, query_seed=6)
    lde = oracle.coset_lde(Z.BABYBEAR, trace, 1)
    layers = oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [lde])
    assert (root == layers[-1][0]).all()
    cw = oracle.combine_columns_ext4(lde, alpha)
    want = oracle.fri_commit_ext4(cw, 3, 42, 5, 10, 6)
    assert (pf.roots == want["roots"]).all() and (pf.final == want["final"]).all()
    assert (pf.query_indices == want["indices"]).all()
    for q in range(10):
        for r in range(pf.rounds):
            assert (pf.query_rows[q, r] == want["queries"][q][r][0]).all()


@pytest.mark.parametrize("log_n,log_final,nq", [(6, 2, 10), (13, 3, 30)])
def test_fri_transcript_matches_oracle(oracle, log_n, log_final, nq):
    """Transcript mode: beta_r drawn after observing root r, the final codeword observed,
    query indices from sample_bits(log_n) — every value equal to the oracle's."""
    cw = rand_field(Z.BABYBEAR, (1 << log_n, 4), 500 + log_n)
    pf = Z.CudaFriProver(42, log_final, nq, transcript=True).commit(cw)
    want = oracle.fri_commit_ext4(cw, log_final, 42, 0, nq, 0, challenger=oracle.DuplexChallenger(0, 42))
    assert (pf.roots == want["roots"]).all() and (pf.betas == want["betas"]).all()
    assert (pf.final == want["final"]).all() and (pf.query_indices == want["indices"]).all()
    for q in range(nq):
        for r in range(pf.rounds):
            row, proof = want["queries"][q][r]
            assert (pf.query_rows[q, r] == row).all()
            assert (pf.siblings(q, r) == np.array(proof).reshape(-1, 8)).all()
    # the seeds play no part in transcript mode
    other = Z.CudaFriProver(42, log_final, nq, challenge_seed=99, query_seed=98, transcript=True).commit(cw)
    assert (other.betas == pf.betas).all() and (other.query_indices == pf.query_indices).all()


def test_pcs_commit_fri_transcript_job(oracle):
    """Commit + FRI with the transcript: alpha is sampled after observing the trace root,
    then the FRI challenges follow from the same transcript."""
    trace = rand_field(Z.BABYBEAR, (1 << 10, 24), 41)
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    root, _, pf = pcs.commit_fri(trace, None, log_final=3, num_queries=12, transcript=True)
    lde = oracle.coset_lde(Z.BABYBEAR, trace, 1)
    layers = oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [lde])
    assert (root == layers[-1][0]).all()
    ch = oracle.DuplexChallenger(0, 42)
    ch.observe(layers[-1][0])
    alpha = ch.sample(4).astype(np.uint32)
    assert (pf.alpha == alpha).all()
    want = oracle.fri_commit_ext4(oracle.combine_columns_ext4(lde, alpha), 3, 42, 0, 12, 0, challenger=ch)
    assert (pf.roots == want["roots"]).all() and (pf.betas == want["betas"]).all()
    assert (pf.final == want["final"]).all() and (pf.query_indices == want["indices"]).all()
    # the same job through the serving engine
    eng = Z.CommitEngine(slots=2)
    r2, pf2, _ = eng.wait(eng.submit(trace, fri={"log_final": 3, "num_queries": 12, "transcript": True}))
    eng.close()
    assert (r2 == root).all() and (pf2.alpha == alpha).all() and (pf2.roots == pf.roots).all()
    assert (pf2.query_indices == pf.query_indices).all()
