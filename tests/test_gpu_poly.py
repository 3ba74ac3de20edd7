"""PolyOpsAccelerator (batch evaluation, coset evaluation, opening quotient) against the
oracle, on the shapes of the reference's own tests (zkf-metal/src/poly.rs:286-400)."""
import numpy as np
import pytest

import ziros_b200 as Z
from conftest import GL_P, rand_field

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops():
    o = Z.CudaPolyOps.new()
    assert o is not None
    return o


def test_poly_eval_reference_shape(oracle, ops):
    coeffs = np.array([(i * 7 + 1) % GL_P for i in range(64)], np.uint64)
    points = np.array([(i * 13 + 3) % GL_P for i in range(2048)], np.uint64)
    assert (ops.batch_eval_goldilocks(coeffs, points) == oracle.poly_eval_gl(coeffs, points)).all()


@pytest.mark.parametrize("n_coeffs,n_points", [(1, 5), (257, 1000), (3, 1)])
def test_poly_eval_random(oracle, ops, n_coeffs, n_points):
    c, x = rand_field(Z.GOLDILOCKS, n_coeffs, n_coeffs), rand_field(Z.GOLDILOCKS, n_points, n_points)
    assert (ops.batch_eval_goldilocks(c, x) == oracle.poly_eval_gl(c, x)).all()


def test_coset_eval_reference_shape(oracle, ops):
    coeffs = np.array([(i * 5 + 9) % GL_P for i in range(1 << 11)], np.uint64)
    got = ops.coset_eval_goldilocks(coeffs, 7, 11)
    # all 2^11 points by Horner in Python is slow: the DFT identity on a sample, plus the oracle's DFT
    shifted = np.array([int(c) * pow(7, i, GL_P) % GL_P for i, c in enumerate(coeffs)], np.uint64)
    want = oracle.dft_batch(Z.GOLDILOCKS, shifted)
    assert (got == want.reshape(-1)).all()
    sample = [0, 1, 1000, 2047]
    direct = oracle.poly_eval_gl(coeffs, [(7 * pow(int(oracle.two_adic_generator(1, 11)), i, GL_P)) % GL_P
                                          for i in sample])
    assert (got[sample] == direct).all()


def test_quotient_reference_shape(oracle, ops):
    coeffs = np.array([(i * 17 + 4) % GL_P for i in range(64)], np.uint64)
    log_n = 11
    w = int(oracle.two_adic_generator(1, log_n))
    pts = [pow(w, i, GL_P) for i in range(1 << log_n)]
    evals = oracle.poly_eval_gl(coeffs, pts)
    f_z = int(oracle.poly_eval_gl(coeffs, [9])[0])
    got = ops.quotient_goldilocks(evals, 9, f_z)
    assert (got == oracle.poly_quotient_gl(evals, 9, f_z)).all()


def test_quotient_with_z_on_the_subgroup(oracle, ops):
    """A point z of the subgroup makes one denominator vanish: that output is 0 and the
    batch inversion around it is unaffected."""
    log_n = 10
    w = int(oracle.two_adic_generator(1, log_n))
    evals = rand_field(Z.GOLDILOCKS, 1 << log_n, 5)
    for k in (0, 7, 15, 16, 1023):
        z = pow(w, k, GL_P)
        got = ops.quotient_goldilocks(evals, z, 12345)
        assert got[k] == 0 and (got == oracle.poly_quotient_gl(evals, z, 12345)).all()
