"""The runtime dispatch driver: a graph of prover nodes over device buffer slots.

Every node's output equals the same operation through its own entry point (itself
pinned to the oracle); a node below a threshold comes back as the fallback node."""
import numpy as np
import pytest

import ziros_b200 as Z
from ziros_b200 import _native as N
from conftest import rand_field

pytestmark = pytest.mark.gpu


def test_lde_merkle_fri_query_graph(oracle):
    rt = Z.ProverRuntime()
    R = Z.ProverRuntime
    trace = rand_field(Z.BABYBEAR, (1 << 10, 24), 61)
    s_tr, s_lde, s_root = rt.buffer(trace.nbytes), rt.buffer(trace.nbytes * 2), rt.buffer(32)
    rt.write(s_tr, trace)
    lde = rt.add(R.LDE, log_n=10, width=24, log_blowup=1, in_slot=s_tr, out_slot=s_lde)
    mk = rt.add(R.MERKLE, deps=[lde], log_n=11, width=24, in_slot=s_lde, out_slot=s_root)
    # FRI: fold an F_p^4 codeword, commit the folded layer as sibling pairs, open queries
    cw = rand_field(Z.BABYBEAR, (1 << 9, 4), 62)
    beta = rand_field(Z.BABYBEAR, 4, 63)
    s_cw, s_fold = rt.buffer(cw.nbytes), rt.buffer(cw.nbytes // 2)
    rt.write(s_cw, cw)
    fold = rt.add(R.FRI_FOLD, log_n=9, in_slot=s_cw, out_slot=s_fold, ext4=True, beta=beta)
    mk2 = rt.add(R.MERKLE, deps=[fold], log_n=7, width=8, in_slot=s_fold)
    idx = np.array([0, 5, 127, 64], np.uint64)
    s_idx, s_open = rt.buffer(idx.nbytes), rt.buffer(len(idx) * (8 + 7 * 8) * 4)
    rt.write(s_idx, idx)
    q = rt.add(R.FRI_QUERY_OPEN, deps=[mk2], count=len(idx), in_slot=s_idx, out_slot=s_open, tree_node=mk2)
    assert rt.execute() is None
    want_lde = oracle.coset_lde(Z.BABYBEAR, trace, 1)
    assert (rt.read(s_lde, want_lde.shape, np.uint32) == want_lde).all()
    layers = oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [want_lde])
    assert (rt.read(s_root, 8, np.uint32) == layers[-1][0]).all()
    folded = oracle.fri_fold_ext4(cw, beta)
    assert (rt.read(s_fold, folded.shape, np.uint32) == folded).all()
    mat = folded.reshape(-1, 8)
    flayers = oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [mat])
    opened = rt.read(s_open, (len(idx), 8 + 7 * 8), np.uint32)
    for k, i in enumerate(idx):
        rows, proof = oracle.mmcs_open(flayers, [mat], int(i))
        assert (opened[k, :8] == rows[0]).all() and (opened[k, 8:] == np.concatenate(proof)).all()
    assert all(rt.node_ms(n) >= 0 for n in (lde, mk, fold, mk2, q))


def test_query_index_past_the_tree_is_an_error():
    """Query indices come from a device buffer; one past the tree is reported (query
    number, index, tree height) instead of opening some other row."""
    rt = Z.ProverRuntime()
    R = Z.ProverRuntime
    m = rand_field(Z.BABYBEAR, (1 << 6, 8), 64)
    s_m = rt.buffer(m.nbytes)
    rt.write(s_m, m)
    mk = rt.add(R.MERKLE, log_n=6, width=8, in_slot=s_m)
    idx = np.array([3, 63, 64, 7], np.uint64)
    s_idx, s_open = rt.buffer(idx.nbytes), rt.buffer(len(idx) * (8 + 6 * 8) * 4)
    rt.write(s_idx, idx)
    rt.add(R.FRI_QUERY_OPEN, deps=[mk], count=len(idx), in_slot=s_idx, out_slot=s_open, tree_node=mk)
    with pytest.raises(Z.ZkbError) as e:
        rt.execute()
    assert e.value.code == N.ERR_INVALID and "query 2 opens row 64 of a 64-row tree" in str(e.value)


def test_ntt_and_poseidon_nodes(oracle):
    rt = Z.ProverRuntime()
    R = Z.ProverRuntime
    m = rand_field(Z.GOLDILOCKS, (1 << 9, 5), 70)
    states = rand_field(Z.GOLDILOCKS, 16 * 300, 71)
    s_m, s_st = rt.buffer(m.nbytes), rt.buffer(states.nbytes)
    rt.write(s_m, m)
    rt.write(s_st, states)
    rt.add(R.NTT, field=Z.GOLDILOCKS, log_n=9, width=5, in_slot=s_m)
    rt.add(R.POSEIDON_BATCH, field=Z.GOLDILOCKS, count=300, in_slot=s_st, seed=42)
    assert rt.execute() is None
    assert (rt.read(s_m, m.shape, np.uint64) == oracle.dft_batch(Z.GOLDILOCKS, m)).all()
    rc, ne, ni = oracle.round_constants(Z.GOLDILOCKS, 42)
    assert (rt.read(s_st, states.shape, np.uint64) == oracle.permute(Z.GOLDILOCKS, states, rc, ne, ni)).all()


def test_fallback_signal_names_the_declined_node():
    rt = Z.ProverRuntime()
    R = Z.ProverRuntime
    s = rt.buffer(1 << 20)
    rt.add(R.POSEIDON_BATCH, count=1000, in_slot=s)
    small = rt.add(R.NTT, log_n=8, width=4, in_slot=s)
    try:
        N.set_thresholds(ntt=1 << 10)
        assert rt.execute() == small
    finally:
        N.set_thresholds()
    assert rt.execute() is None


def test_nodes_may_only_depend_on_earlier_nodes():
    rt = Z.ProverRuntime()
    with pytest.raises(Z.ZkbError):
        rt.add(Z.ProverRuntime.NTT, deps=[0], log_n=4, width=1, in_slot=rt.buffer(64))


def test_merkle_node_tree_opens_like_a_plain_tree(oracle):
    rt = Z.ProverRuntime()
    m = rand_field(Z.BABYBEAR, (1 << 8, 12), 80)
    s = rt.buffer(m.nbytes)
    rt.write(s, m)
    node = rt.add(Z.ProverRuntime.MERKLE, log_n=8, width=12, in_slot=s)
    assert rt.execute() is None
    mmcs = Z.CudaMerkleTreeMmcs(Z.BABYBEAR, 42)
    layers = oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [m])
    rows, sib = mmcs.open_batch(77, rt.tree(node, 1 << 8, 12))
    want_rows, want_sib = oracle.mmcs_open(layers, [m], 77)
    assert (rows[0] == want_rows[0]).all() and all((a == b).all() for a, b in zip(sib, want_sib))
    assert mmcs.verify_batch(layers[-1][0], [(1 << 8, 12)], 77, rows, sib)
