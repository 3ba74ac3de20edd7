"""Poseidon2 MMCS on the GPU vs the oracle (bit-exact roots, layers and openings).

Mirrors zkf-metal/src/merkle.rs:714-799 (BabyBear 4096 x 4, seed 42, against p3's
MerkleTreeMmcs) and the vendored MMCS tests (mixed heights, odd heights,
openings: vendor/p3-merkle-tree-gpu/src/mmcs.rs:368-710), with every row width —
the reference's Metal path only hashes rows of at most 8 elements."""
import numpy as np
import pytest

import ziros_b200 as Z
from conftest import rand_field

pytestmark = pytest.mark.gpu


def check_tree(oracle, field, seed, mats, width=16):
    mmcs = Z.CudaMerkleTreeMmcs(field, seed, width)
    root, tree = mmcs.commit(mats)
    layers = oracle.mmcs_commit(oracle.hasher(field, seed, width), mats)
    got = tree.digest_layers()
    assert len(got) == len(layers)
    for a, b in zip(got, layers):
        assert a.shape == b.shape and (a == b).all()
    assert (root == layers[-1][0]).all()
    return mmcs, tree, layers


def test_reference_shape_babybear_4096x4(oracle):
    m = rand_field(Z.BABYBEAR, (4096, 4), 42)
    check_tree(oracle, Z.BABYBEAR, 42, [m])


@pytest.mark.parametrize("field", [Z.BABYBEAR, Z.GOLDILOCKS])
@pytest.mark.parametrize("width", [1, 7, 8, 9, 16, 17, 33, 64, 256])
def test_widths(oracle, field, width):
    m = rand_field(field, (1 << 9, width), width)
    check_tree(oracle, field, 11, [m])


@pytest.mark.parametrize("height", [1, 2, 3, 5, 6, 7, 100, 1023, 1025])
def test_heights(oracle, height):
    m = rand_field(Z.BABYBEAR, (height, 10), height)
    check_tree(oracle, Z.BABYBEAR, 3, [m])


def test_mixed_heights_injection(oracle):
    for field in (Z.BABYBEAR, Z.GOLDILOCKS):
        mats = [rand_field(field, (64, 5), 1), rand_field(field, (256, 3), 2), rand_field(field, (256, 9), 3),
                rand_field(field, (16, 12), 4), rand_field(field, (2, 2), 5)]
        check_tree(oracle, field, 99, mats)
        # non power-of-two heights obeying ceil(max / 2^k)
        mats = [rand_field(field, (100, 4), 6), rand_field(field, (50, 6), 7), rand_field(field, (13, 1), 8)]
        check_tree(oracle, field, 98, mats)


def test_rejects_incompatible_heights():
    mmcs = Z.CudaMerkleTreeMmcs(Z.BABYBEAR, 1)
    with pytest.raises(Z.ZkbError):
        mmcs.commit([rand_field(0, (8, 2), 1), rand_field(0, (6, 2), 2)])


def test_goldilocks_width12_hasher(oracle):
    m = rand_field(Z.GOLDILOCKS, (1 << 10, 64), 12)
    _, tree, _ = check_tree(oracle, Z.GOLDILOCKS, 12, [m], width=12)
    assert tree.digest_elems == 4


def test_open_batch(oracle):
    field = Z.GOLDILOCKS
    mats = [rand_field(field, (128, 6), 1), rand_field(field, (32, 3), 2)]
    mmcs, tree, layers = check_tree(oracle, field, 5, mats)
    for idx in (0, 1, 77, 127):
        rows, proof = mmcs.open_batch(idx, tree)
        want_rows, want_proof = oracle.mmcs_open(layers, mats, idx)
        assert all((a == b).all() for a, b in zip(rows, want_rows))
        assert len(proof) == len(want_proof) and all((a == b).all() for a, b in zip(proof, want_proof))
    with pytest.raises(Z.ZkbError):
        mmcs.open_batch(128, tree)


def test_commit_device_resident(oracle):
    import torch

    m = rand_field(Z.BABYBEAR, (1 << 12, 32), 8)
    t = torch.from_numpy(m.view(np.int32)).cuda()
    mmcs = Z.CudaMerkleTreeMmcs(Z.BABYBEAR, 8)
    root, tree = mmcs.commit_dev([t])
    layers = oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 8), [m])
    assert (root == layers[-1][0]).all()
    rows, _ = mmcs.open_batch(5, tree)
    assert (rows[0] == m[5]).all()


def test_config1_lde_commit_root(oracle):
    """BabyBear 2^14 x 16 -> coset LDE blowup 2 (bit-reversed rows) -> W16 MMCS root."""
    t = rand_field(Z.BABYBEAR, (1 << 14, 16), 1)
    lde = Z.CudaDft(Z.BABYBEAR).coset_lde_batch(t, 1, bit_reverse_rows=True)
    want_lde = oracle.coset_lde(Z.BABYBEAR, t, 1)
    assert (lde == want_lde).all()
    root, _ = Z.CudaMerkleTreeMmcs(Z.BABYBEAR, 42).commit([lde])
    layers = oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [want_lde])
    assert (root == layers[-1][0]).all()
