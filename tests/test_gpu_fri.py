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
