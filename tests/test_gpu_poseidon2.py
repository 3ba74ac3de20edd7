"""Poseidon2 batch permutation on the GPU vs the oracle (bit-exact).

Mirrors the reference's differential tests (zkf-metal/src/poseidon2/mod.rs:507-750:
2000 random states against p3, patterned states) and its golden vector
(zkf-backends/src/wrapping/poseidon2_goldilocks.rs:538-620)."""
import json
import os

import numpy as np
import pytest

import ziros_b200 as Z
from conftest import BB_P, GL_P, rand_field

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))


@pytest.fixture(scope="module")
def p2():
    p = Z.CudaPoseidon2.new()
    assert p is not None, "no CUDA device"
    return p


def test_golden_vector_on_gpu(p2):
    g = GOLD["poseidon2_goldilocks_w16_seed42"]
    rc, ne, ni = Z.round_constants(Z.GOLDILOCKS, g["seed"])
    st = np.array(g["input"], dtype=np.uint64)
    assert p2.batch_permute_goldilocks(st, rc, ne, ni)
    assert [int(x) for x in st] == [int(h, 16) for h in g["output_hex"]]


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("seed", [42, 7, 19])
def test_batch_matches_oracle(oracle, p2, field, seed):
    rc, ne, ni = Z.round_constants(field, seed)
    states = rand_field(field, (2000, 16), seed)
    want = oracle.permute(field, states, rc, ne, ni)
    got = states.copy()
    fn = p2.batch_permute_babybear if field == Z.BABYBEAR else p2.batch_permute_goldilocks
    assert fn(got, rc, ne, ni)
    assert (got == want).all()


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
def test_edge_values(oracle, p2, field):
    p = BB_P if field == Z.BABYBEAR else GL_P
    dt = np.uint32 if field == Z.BABYBEAR else np.uint64
    vals = np.array([0, 1, 2, p - 1, p - 2, p // 2, (p + 1) // 2], dtype=dt)
    states = np.resize(vals, (64, 16)).astype(dt)
    states[1::2] = states[1::2][:, ::-1]
    rc, ne, ni = Z.round_constants(field, 3)
    want = oracle.permute(field, states, rc, ne, ni)
    got = states.copy()
    fn = p2.batch_permute_babybear if field == Z.BABYBEAR else p2.batch_permute_goldilocks
    assert fn(got, rc, ne, ni)
    assert (got == want).all()


def test_nonstandard_round_counts(oracle, p2):
    rc_full, _, _ = Z.round_constants(Z.GOLDILOCKS, 5)
    # 4 external (2 + 2) and 3 internal rounds: the looped kernel path
    rc = np.concatenate([rc_full[:32], rc_full[128:131], rc_full[32:64]])
    states = rand_field(Z.GOLDILOCKS, (100, 16), 5)
    want = oracle.permute(Z.GOLDILOCKS, states, rc, 4, 3)
    got = states.copy()
    assert p2.batch_permute_goldilocks(got, rc, 4, 3)
    assert (got == want).all()


def test_invalid_arguments_raise(p2):
    rc, ne, ni = Z.round_constants(Z.BABYBEAR, 1)
    with pytest.raises(Z.ZkbError) as e:
        p2.batch_permute_babybear(np.zeros(16, np.uint32), rc[:-1], ne, ni)
    assert e.value.code == -1
    with pytest.raises(Z.ZkbError):
        p2.batch_permute_babybear(np.zeros(15, np.uint32), rc, ne, ni)
    bad = rc.copy()
    bad[0] = BB_P  # not canonical
    with pytest.raises(Z.ZkbError):
        p2.batch_permute_babybear(np.zeros(16, np.uint32), bad, ne, ni)


def test_empty_batch(p2):
    rc, ne, ni = Z.round_constants(Z.BABYBEAR, 1)
    assert p2.batch_permute_babybear(np.zeros(0, np.uint32), rc, ne, ni)


def test_device_resident_form(oracle, p2):
    import torch

    rc, ne, ni = Z.round_constants(Z.BABYBEAR, 9)
    states = rand_field(Z.BABYBEAR, (4096, 16), 9)
    t = torch.from_numpy(states.view(np.int32).copy()).cuda()
    p2.batch_permute_dev(Z.BABYBEAR, t, rc, ne, ni)
    got = t.cpu().numpy().view(np.uint32)
    assert (got == oracle.permute(Z.BABYBEAR, states, rc, ne, ni)).all()
