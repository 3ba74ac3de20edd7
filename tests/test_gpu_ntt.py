"""DFT / coset LDE on the GPU vs the oracle (bit-exact).

Mirrors zkf-metal/src/ntt/p3_adapter.rs:604-769 (known answer, 2^13 single and
multi-column, forward->inverse round trip, patterned seeds 5/23 with widths 1/4)
and adds the coset LDE that TwoAdicFriPcs::commit runs, at the configured sizes
and through size-independent properties at the full Goldilocks 2^20 x 64 size."""
import numpy as np
import pytest

import ziros_b200 as Z
from conftest import BB_P, GL_P, rand_field

pytestmark = pytest.mark.gpu


def patterned(field, h, w, seed):
    """The reference's patterned_{goldilocks,babybear}_values (p3_adapter.rs:581-602)."""
    i = np.arange(h * w, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _patterned(field, h, w, seed, i)


def _patterned(field, h, w, seed, i):
    if field == Z.GOLDILOCKS:
        v = np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + i * np.uint64(0xBF58476D1CE4E5B9)
        v = np.where(v >= np.uint64(GL_P), v - np.uint64(GL_P), v)
        return v.reshape(h, w)
    v = np.uint64(seed) * np.uint64(0xDA942042E4DD58B5) + i * np.uint64(0x94D049BB133111EB)
    return (v % np.uint64(BB_P)).astype(np.uint32).reshape(h, w)


def test_dft_known_answer():
    out = Z.CudaDft(Z.GOLDILOCKS).dft_batch(np.array([1, 2, 3, 4], np.uint64))
    assert int(out[0, 0]) == 10


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("seed,width", [(5, 1), (23, 4), (0, 16), (0, 27)])
def test_dft_matches_oracle(oracle, field, seed, width):
    m = patterned(field, 1 << 13, width, seed) if seed else rand_field(field, (1 << 13, width), 3)
    dft = Z.CudaDft(field)
    got = dft.dft_batch(m)
    assert (got == oracle.dft_batch(field, m)).all()
    assert (dft.idft_batch(got) == m).all()


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("log_h", [1, 2, 7, 11, 12, 17])
def test_dft_sizes(oracle, field, log_h):
    m = rand_field(field, (1 << log_h, 3), log_h)
    got = Z.CudaDft(field).dft_batch(m)
    assert (got == oracle.dft_batch(field, m)).all()


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("log_h,width,log_b", [
    (0, 3, 1), (1, 1, 1), (3, 5, 3), (5, 7, 2), (10, 16, 1), (13, 8, 2), (14, 16, 1), (12, 24, 3),
    (16, 2, 1),
    # widths that are not a multiple of the column chunk: bulk + 8/4/1-column remainders
    (12, 31, 1), (13, 29, 1), (11, 45, 2), (15, 13, 1)])
def test_coset_lde_matches_oracle(oracle, field, log_h, width, log_b):
    t = rand_field(field, (1 << log_h, width), 1000 + log_h * 10 + log_b)
    got = Z.CudaDft(field).coset_lde_batch(t, log_b, bit_reverse_rows=True)
    assert (got == oracle.coset_lde(field, t, log_b)).all()


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
def test_coset_lde_natural_order_and_shift(oracle, field):
    t = rand_field(field, (1 << 9, 6), 77)
    dft = Z.CudaDft(field)
    nat = dft.coset_lde_batch(t, 2, shift=5, bit_reverse_rows=False)
    assert (nat == oracle.coset_lde(field, t, 2, shift=5, bitrev=False)).all()


def test_lde_config1_babybear(oracle):
    """BabyBear 2^14 x 16, blowup 2, bit-reversed rows: every value bit-exact."""
    t = rand_field(Z.BABYBEAR, (1 << 14, 16), 2024)
    got = Z.CudaDft(Z.BABYBEAR).coset_lde_batch(t, 1, bit_reverse_rows=True)
    assert (got == oracle.coset_lde(Z.BABYBEAR, t, 1)).all()


def test_lde_goldilocks_full_size_columns(oracle):
    """Goldilocks 2^20 x 64, blowup 4 -> 2^22 rows.  Four whole columns are compared
    bit-exactly with the oracle (columns are independent transforms); the other 60
    are checked by the size-independent property that the inverse DFT of each LDE
    column (natural order) vanishes above degree n."""
    import torch

    n, w, lb = 1 << 20, 64, 2
    t = rand_field(Z.GOLDILOCKS, (n, w), 42)
    dft = Z.CudaDft(Z.GOLDILOCKS)
    tt = torch.from_numpy(t.view(np.int64)).cuda()
    out = torch.empty((n << lb, w), dtype=torch.int64, device="cuda")
    dft.coset_lde_batch_dev(tt, lb, out, bit_reverse_rows=True)
    torch.cuda.synchronize()
    lde = out.cpu().numpy().view(np.uint64)
    cols = [0, 17, 38, 63]
    want = oracle.coset_lde(Z.GOLDILOCKS, np.ascontiguousarray(t[:, cols]), lb)
    assert (lde[:, cols] == want).all()
    # degree bound on every column: natural order row r sits at bit-reversed position rev(r)
    bits = 22
    x = np.arange(n << lb, dtype=np.int64)
    r = np.zeros_like(x)
    for b in range(bits):
        r |= ((x >> b) & 1) << (bits - 1 - b)
    coef = dft.idft_batch(lde[r])
    assert not coef[n:].any()
    # the low coefficients are the trace's, scaled by shift^m
    assert coef[:n].any()


def test_ntt_accelerator_name_and_availability():
    """zkf-metal/src/ntt/mod.rs:114-120 (metal_ntt_accelerator_available)."""
    acc = Z.CudaNttAccelerator.new()
    assert acc is not None and acc.name() == "cuda-b200-ntt" and acc.is_available()
    assert acc.max_log_size() == 26


def test_ntt_accelerator_forward_inverse_roundtrip(oracle):
    """zkf-metal/src/ntt/mod.rs:122-145: values 1..2^13 forward then inverse; the forward
    result is also compared with the oracle's width-1 Goldilocks DFT (the call the
    NttAccelerator shim makes: zkb_dft_batch(GOLDILOCKS, ..., width 1, inverse))."""
    acc = Z.CudaNttAccelerator()
    n = 1 << 13
    values = [i + 1 for i in range(n)]
    original = list(values)
    acc.forward_ntt(values)
    assert values != original
    want = oracle.dft_batch(Z.GOLDILOCKS, np.arange(1, n + 1, dtype=np.uint64).reshape(-1, 1))
    assert values == [int(x) for x in want[:, 0]]
    acc.inverse_ntt(values)
    assert values == original


def test_ntt_accelerator_reduces_inputs_and_rejects_bad_sizes(oracle):
    """Inputs above p are taken mod p after truncation to 64 bits (Goldilocks::from_u64 of
    the low 8 bytes); sizes that are not powers of two are errors, as in the reference."""
    acc = Z.CudaNttAccelerator()
    big = [GL_P + 5, (1 << 64) + 3, GL_P - 1, 0]
    acc.forward_ntt(big)
    want = oracle.dft_batch(Z.GOLDILOCKS, np.array([5, 3, GL_P - 1, 0], np.uint64).reshape(-1, 1))
    assert big == [int(x) for x in want[:, 0]]
    with pytest.raises(Z.ZkbError):
        acc.forward_ntt([1, 2, 3])
    with pytest.raises(Z.ZkbError):
        acc.inverse_ntt([])
