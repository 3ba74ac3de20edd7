"""NTT tiles with tensor-copy (TMA) loads against register loads: the same outputs, bit
for bit.

Tile-load mode 1 (the default) makes every pass and fused LDE middle whose rows and
column chunks are multiples of 16 bytes (BabyBear: width a multiple of 4, chunks of 4
columns or more; Goldilocks: even width, chunks of 4 or 8) bring its tile into shared
memory with one cp.async.bulk.tensor copy; the rest keep the coalesced loads (mode 0 uses
those everywhere).  Each case runs both ways and against the oracle, and checks that no
copy's bounded wait gave up."""
import numpy as np
import pytest

import ziros_b200 as Z
from ziros_b200 import _native as N
from conftest import rand_field

pytestmark = pytest.mark.gpu


@pytest.fixture
def tma_mode():
    N.ntt_tile_load_errors()  # start from a clear count
    yield
    N.set_ntt_tile_loads(1)  # the default


def _both(fn):
    N.set_ntt_tile_loads(0)
    a = fn()
    N.set_ntt_tile_loads(1)
    b = fn()
    assert N.ntt_tile_load_errors() == 0
    return a, b


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("log_h,width", [(1, 4), (5, 8), (10, 16), (11, 4), (13, 20), (17, 24), (20, 16),
                                         (14, 27), (12, 3), (9, 2), (15, 14)])
def test_dft_tile_loads_agree(oracle, tma_mode, field, log_h, width):
    m = rand_field(field, (1 << log_h, width), 300 + log_h)
    dft = Z.CudaDft(field)
    a, b = _both(lambda: dft.dft_batch(m))
    assert (a == b).all()
    if log_h <= 14:
        assert (b == oracle.dft_batch(field, m)).all()
    ia, ib = _both(lambda: dft.idft_batch(a))
    assert (ia == m).all() and (ib == m).all()


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("log_h,width,log_b", [(14, 16, 1), (12, 64, 2), (18, 32, 1), (13, 36, 3), (16, 8, 1),
                                               (11, 10, 2)])
def test_coset_lde_tile_loads_agree(oracle, tma_mode, field, log_h, width, log_b):
    t = rand_field(field, (1 << log_h, width), 400 + log_h)
    dft = Z.CudaDft(field)
    a, b = _both(lambda: dft.coset_lde_batch(t, log_b, bit_reverse_rows=True))
    assert (a == b).all()
    if log_h <= 14:
        assert (b == oracle.coset_lde(field, t, log_b)).all()


@pytest.mark.parametrize("field,p2w,log_b", [(Z.BABYBEAR, 16, 1), (Z.GOLDILOCKS, 12, 2)])
def test_commit_root_with_tile_loads(tma_mode, field, p2w, log_b):
    t = rand_field(field, (1 << 16, 64), 501)
    pcs = Z.CudaTwoAdicPcs(field, 42, log_b, p2w)
    a, b = _both(lambda: pcs.commit(t)[0])
    assert (a == b).all()


def test_tile_load_mode_rejects_unknown():
    with pytest.raises(N.ZkbError):
        N.set_ntt_tile_loads(2)
