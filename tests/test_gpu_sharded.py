"""The commitment split over ranks (ziros_b200.sharded) with the CUDA per-rank compute.

One GPU is available to these tests, so the ranks are processes on cuda:0: one rank over
NCCL, and two ranks over gloo (the exchange staged through host memory).  No kernel of
one rank waits on another rank's; the ranks meet only in host-side collectives.  The
result must equal the single-device commitment (zkb_pcs_commit_fri / zkb_pcs_commit)
of the whole trace: root, openings and FRI proof."""
import os
import pickle
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from ziros_b200 import accel as A  # noqa: E402
from ziros_b200 import sharded as S  # noqa: E402

pytestmark = pytest.mark.gpu

BB, GL = A.BABYBEAR, A.GOLDILOCKS
BB_P, GL_P = 0x78000001, 0xFFFFFFFF00000001


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _trace(field, log_h, width, seed):
    g = np.random.default_rng(seed)
    if field == BB:
        return g.integers(0, BB_P, size=(1 << log_h, width), dtype=np.uint32)
    return g.integers(0, GL_P, size=(1 << log_h, width), dtype=np.uint64)


def _indices(log_n):
    n = 1 << log_n
    return sorted({0, 1, n // 2 - 1, n // 2, n - 1, (n * 5) // 11})


def _worker(rank, world, port, backend, out_dir, case):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    kw = {"device_id": torch.device("cuda", 0)} if backend == "nccl" else {}
    dist.init_process_group(backend, rank=rank, world_size=world, **kw)
    try:
        field, log_h, width, log_blowup, p2w, fri = case
        trace = _trace(field, log_h, width, 11)
        c0, c1 = S.column_ranges(width, world)[rank]
        dt = torch.int32 if field == BB else torch.int64
        cols = torch.from_numpy(np.ascontiguousarray(trace[:, c0:c1]).view(
            np.int32 if field == BB else np.int64)).to("cuda:0")
        ops = S.CudaShardOps(field, 42, log_blowup, p2w)
        res = S.commit_sharded(cols, width, ops, fri=fri)
        assert res.block.dtype == dt
        out = {"root": res.root, "openings": {i: res.open(i) for i in _indices(res.log_n)}}
        if res.fri is not None:
            p = res.fri
            out["fri"] = {"roots": p.roots, "betas": p.betas, "final": p.final, "indices": p.query_indices,
                          "rows": p.query_rows, "siblings": p.query_siblings}
            out["alpha"] = res.alpha
        torch.cuda.synchronize()
        with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump(out, f)
        del res
        dist.barrier()
    finally:
        dist.destroy_process_group()


CASES = {
    "bb_seeded_fri": (BB, 12, 24, 1, 16, S.FriArgs(log_final=3, num_queries=10, alpha=[5, 6, 7, 8],
                                                   challenge_seed=3, query_seed=8)),
    "bb_transcript_fri": (BB, 11, 17, 1, 16, S.FriArgs(log_final=2, num_queries=6, transcript=True)),
    "gl_w16": (GL, 10, 10, 2, 16, None),
    "gl_w12": (GL, 9, 7, 1, 12, None),
}


@pytest.mark.parametrize("world,backend,name", [
    (1, "nccl", "bb_seeded_fri"), (2, "gloo", "bb_seeded_fri"), (2, "gloo", "bb_transcript_fri"),
    (1, "nccl", "gl_w16"), (2, "gloo", "gl_w12")])
def test_sharded_commit_equals_single_device_commit(world, backend, name, tmp_path):
    case = CASES[name]
    mp.spawn(_worker, args=(world, _free_port(), backend, str(tmp_path), case), nprocs=world, join=True)
    res = [pickle.load(open(tmp_path / f"rank{r}.pkl", "rb")) for r in range(world)]

    field, log_h, width, log_blowup, p2w, fri = case
    trace = _trace(field, log_h, width, 11)
    pcs = A.CudaTwoAdicPcs(field, 42, log_blowup, p2w)
    if fri is None:
        root, tree = pcs.commit(trace)
        proof = None
    else:
        root, tree, proof = pcs.commit_fri(trace, fri.alpha, fri.log_final, fri.num_queries, fri.challenge_seed,
                                           fri.query_seed, want_tree=True, transcript=fri.transcript)
    for r in res:
        assert np.array_equal(r["root"], root)
        for i, (row, sibs) in r["openings"].items():
            rows_ref, sibs_ref = pcs.mmcs.open_batch(i, tree)
            assert np.array_equal(row, rows_ref[0]), i
            assert len(sibs) == len(sibs_ref) and all(np.array_equal(a, b) for a, b in zip(sibs, sibs_ref)), i
        if proof is not None:
            assert np.array_equal(r["alpha"], proof.alpha)
            f = r["fri"]
            assert np.array_equal(f["roots"], proof.roots) and np.array_equal(f["betas"], proof.betas)
            assert np.array_equal(f["final"], proof.final)
            assert np.array_equal(f["indices"], proof.query_indices)
            assert np.array_equal(f["rows"], proof.query_rows)
            assert np.array_equal(f["siblings"], proof.query_siblings)


def test_fri_with_a_caller_challenger_matches_the_transcript_job():
    """zkb_fri_commit_babybear_ext4_challenger_dev continues the caller's transcript: a
    challenger that observed the root and drew alpha gives the commit+FRI job's proof."""
    trace = _trace(BB, 10, 12, 5)
    pcs = A.CudaTwoAdicPcs(BB, 42, 1)
    root, tree, proof = pcs.commit_fri(trace, None, 2, 7, want_tree=True, transcript=True)
    ch = A.Challenger(BB, 42)
    ch.observe(root.astype(np.uint64))
    alpha = ch.sample(4).astype(np.uint32)
    assert np.array_equal(alpha, proof.alpha)
    lde = torch.from_numpy(A.CudaDft(BB).coset_lde_batch(trace, 1, bit_reverse_rows=True).view(np.int32)).cuda()
    cw = torch.empty((lde.shape[0], 4), dtype=torch.int32, device="cuda")
    A.combine_columns_dev(lde, alpha, cw)
    p2 = A.CudaFriProver(42, 2, 7).commit_dev(cw, ch)
    assert np.array_equal(p2.roots, proof.roots) and np.array_equal(p2.betas, proof.betas)
    assert np.array_equal(p2.query_indices, proof.query_indices)
    assert np.array_equal(p2.query_siblings, proof.query_siblings)
    # the challenger moved on: its next sample is what the transcript draws after the queries
    assert ch.sample(1).shape == (1,)


def test_compress_matches_the_tree_levels():
    trace = _trace(GL, 6, 5, 2)
    for p2w in (16, 12):
        mmcs = A.CudaMerkleTreeMmcs(GL, 42, p2w)
        root, tree = mmcs.commit([trace])
        layers = tree.digest_layers()
        for l in range(len(layers) - 1):
            got = mmcs.compress(layers[l][0::2], layers[l][1::2])
            assert np.array_equal(got, layers[l + 1])


def test_one_rank_without_a_process_group():
    """commit_sharded with no process group: the whole trace on this device."""
    assert not dist.is_initialized()
    field, log_h, width, log_blowup, p2w, fri = CASES["bb_seeded_fri"]
    trace = _trace(field, log_h, width, 11)
    ops = S.CudaShardOps(field, 42, log_blowup, p2w)
    res = S.commit_sharded(torch.from_numpy(trace.view(np.int32)).cuda(), width, ops, fri=fri)
    pcs = A.CudaTwoAdicPcs(field, 42, log_blowup, p2w)
    root, tree, proof = pcs.commit_fri(trace, fri.alpha, fri.log_final, fri.num_queries, fri.challenge_seed,
                                       fri.query_seed, want_tree=True)
    assert np.array_equal(res.root, root)
    assert np.array_equal(res.fri.roots, proof.roots) and np.array_equal(res.fri.query_siblings,
                                                                         proof.query_siblings)
    row, sibs = res.open(77)
    rows_ref, sibs_ref = pcs.mmcs.open_batch(77, tree)
    assert np.array_equal(row, rows_ref[0]) and all(np.array_equal(a, b) for a, b in zip(sibs, sibs_ref))


@pytest.mark.parametrize("rows,width", [(1 << 10, 24), (1 << 9, 13), (1, 8), (1 << 8, 256)])
def test_commit_reduce_equals_commit_then_combine(rows, width):
    """zkb_mmcs_commit_reduce_dev: the same tree as zkb_mmcs_commit_dev and the same
    codeword as zkb_combine_columns_babybear_ext4_dev, in one pass."""
    m = torch.from_numpy(_trace(BB, max(rows.bit_length() - 1, 0), width, 9)[:rows].view(np.int32)).cuda()
    alpha = np.array([11, 22, 33, 44], np.uint32)
    mmcs = A.CudaMerkleTreeMmcs(BB, 42)
    root_ref, tree_ref = mmcs.commit_dev([m])
    cw_ref = torch.empty((rows, 4), dtype=torch.int32, device="cuda")
    A.combine_columns_dev(m, alpha, cw_ref)
    cw = torch.zeros((rows, 4), dtype=torch.int32, device="cuda")
    root, tree = mmcs.commit_reduce_dev(m, alpha, cw)
    assert np.array_equal(root, root_ref)
    assert torch.equal(cw, cw_ref)
    for i in sorted({0, rows // 2, rows - 1}):
        a, b = mmcs.open_batch(i, tree), mmcs.open_batch(i, tree_ref)
        assert np.array_equal(a[0][0], b[0][0]) and all(np.array_equal(x, y) for x, y in zip(a[1], b[1]))
