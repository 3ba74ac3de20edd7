"""The commitment split over ranks (ziros_b200.sharded) on CPU gloo ranks.

Each rank holds a column slice of the trace; the per-rank compute is the oracle (an
object with CudaShardOps' methods), so these tests check the exchange: the column split,
the all-to-all of row blocks, the placement of the column blocks, the subtree roots and
top levels, the collective openings and the gathered FRI codeword.  The result must equal
the oracle's single-device pipeline on the whole trace: root, every opening, and the FRI
proof (seeded and transcript)."""
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

import oracle  # noqa: E402
from ziros_b200 import sharded as S  # noqa: E402

BB, GL = oracle.BABYBEAR, oracle.GOLDILOCKS


class OracleShardOps:
    """CudaShardOps' interface over the oracle, on CPU tensors."""

    def __init__(self, field, seed, log_blowup, p2_width=16):
        self.field, self.seed, self.log_blowup = field, seed, log_blowup
        self.device = torch.device("cpu")
        self.dtype = torch.int32 if field == BB else torch.int64
        self.np_dtype = np.uint32 if field == BB else np.uint64
        self.h = oracle.hasher(field, seed, p2_width)
        self.digest_elems = self.h.out

    def _np(self, t):
        return t.contiguous().numpy().view(np.uint32 if t.dtype == torch.int32 else np.uint64)

    def _t(self, a):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(np.int32 if a.dtype == np.uint32 else np.int64).copy())

    def empty(self, rows, cols, ext4=False):
        return torch.empty((rows, cols), dtype=torch.int32 if ext4 else self.dtype)

    def lde(self, cols):
        return self._t(oracle.coset_lde(self.field, self._np(cols), self.log_blowup))

    def commit(self, block):
        mat = self._np(block).copy()
        layers = oracle.mmcs_commit(self.h, [mat])
        return layers[-1][0], (layers, mat)

    def open(self, tree, index):
        layers, mat = tree
        rows, proof = oracle.mmcs_open(layers, [mat], index)
        return rows[0], proof

    def compress(self, left, right):
        return np.stack([oracle.compress(self.h, a, b) for a, b in zip(left, right)])

    def challenger(self):
        return oracle.DuplexChallenger(self.field, self.seed)

    def combine(self, block, alpha):
        return self._t(oracle.combine_columns_ext4(self._np(block), alpha))

    def fri(self, codeword, args, challenger=None):
        return oracle.fri_commit_ext4(self._np(codeword), args.log_final, self.seed, args.challenge_seed,
                                      args.num_queries, args.query_seed, challenger)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _trace(field, log_h, width, seed):
    n = (1 << log_h) * width
    if field == BB:
        return oracle.rng_bb(seed, n).reshape(1 << log_h, width)
    v = oracle.rng_u64(seed, n)
    return (v % np.uint64(oracle.GL_P)).reshape(1 << log_h, width)


def _worker(rank, world, port, out_dir, case):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        field, log_h, width, log_blowup, p2w, fri = case
        trace = _trace(field, log_h, width, 7)
        c0, c1 = S.column_ranges(width, world)[rank]
        ops = OracleShardOps(field, 42, log_blowup, p2w)
        cols = ops._t(np.ascontiguousarray(trace[:, c0:c1]))
        res = S.commit_sharded(cols, width, ops, fri=fri)
        big_n = 1 << res.log_n
        idx = sorted({0, 1, big_n // 2 - 1, big_n // 2, big_n - 1, (big_n * 3) // 7})
        openings = {i: res.open(i) for i in idx}
        out = {"root": res.root, "openings": openings, "block_rows": res.block.shape[0],
               "fri": res.fri, "alpha": res.alpha}
        with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump(out, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _single(case):
    field, log_h, width, log_blowup, p2w, fri = case
    trace = _trace(field, log_h, width, 7)
    h = oracle.hasher(field, 42, p2w)
    lde = oracle.coset_lde(field, trace, log_blowup)
    layers = oracle.mmcs_commit(h, [lde])
    root = layers[-1][0]
    proof, alpha = None, None
    if fri is not None:
        ch = None
        if fri.transcript:
            ch = oracle.DuplexChallenger(field, 42)
            ch.observe(root.astype(np.uint64))
            alpha = ch.sample(4).astype(np.uint32)
        else:
            alpha = np.asarray(fri.alpha, np.uint32)
        cw = oracle.combine_columns_ext4(lde, alpha)
        proof = oracle.fri_commit_ext4(cw, fri.log_final, 42, fri.challenge_seed, fri.num_queries,
                                       fri.query_seed, ch)
    return lde, layers, root, proof, alpha


def _run(world, case, tmp_path):
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path), case), nprocs=world, join=True)
    return [pickle.load(open(tmp_path / f"rank{r}.pkl", "rb")) for r in range(world)]


def _same_fri(a, b):
    assert np.array_equal(a["roots"], b["roots"]) and np.array_equal(a["betas"], b["betas"])
    assert np.array_equal(a["final"], b["final"]) and np.array_equal(a["indices"], b["indices"])
    for qa, qb in zip(a["queries"], b["queries"]):
        for (ra, pa), (rb, pb) in zip(qa, qb):
            assert np.array_equal(ra, rb) and all(np.array_equal(x, y) for x, y in zip(pa, pb))


CASES = {
    # field, log_h, width, log_blowup, Poseidon2 width, FRI
    "bb_seeded_fri": (BB, 7, 13, 1, 16, S.FriArgs(log_final=2, num_queries=5, alpha=[3, 5, 7, 11],
                                                  challenge_seed=9, query_seed=4)),
    "bb_transcript_fri": (BB, 6, 9, 1, 16, S.FriArgs(log_final=1, num_queries=4, transcript=True)),
    "gl_w16": (GL, 6, 10, 2, 16, None),
    "gl_w12_narrow": (GL, 5, 3, 1, 12, None),  # fewer columns than ranks at world 4
}


@pytest.mark.parametrize("world,name", [(2, "bb_seeded_fri"), (4, "bb_seeded_fri"), (2, "bb_transcript_fri"),
                                        (2, "gl_w16"), (4, "gl_w12_narrow")])
def test_sharded_commit_equals_single_device(world, name, tmp_path):
    case = CASES[name]
    res = _run(world, case, tmp_path)
    lde, layers, root, proof, alpha = _single(case)
    field, log_h, width, log_blowup, p2w, fri = case
    for r in res:
        assert np.array_equal(r["root"], root)
        assert r["block_rows"] == lde.shape[0] // world
        for i, (row, sibs) in r["openings"].items():
            rows_ref, sibs_ref = oracle.mmcs_open(layers, [lde], i)
            assert np.array_equal(row, rows_ref[0]), i
            assert len(sibs) == len(sibs_ref) and all(np.array_equal(a, b) for a, b in zip(sibs, sibs_ref)), i
        if fri is not None:
            assert np.array_equal(r["alpha"], alpha)
            _same_fri(r["fri"], proof)


def test_column_ranges_cover_the_width_in_order():
    for width in (1, 3, 13, 256):
        for world in (1, 2, 4, 8):
            rs = S.column_ranges(width, world)
            assert rs[0][0] == 0 and rs[-1][1] == width and len(rs) == world
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(b - a for a, b in rs) - min(b - a for a, b in rs) <= 1


def _bad_world_worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ops = OracleShardOps(BB, 42, 1)
        c0, c1 = S.column_ranges(6, world)[rank]
        msg = ""
        try:
            S.commit_sharded(torch.zeros((8, c1 - c0), dtype=torch.int32), 6, ops)
        except ValueError as e:
            msg = str(e)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(msg)
    finally:
        dist.destroy_process_group()


def test_non_power_of_two_world_is_rejected_before_any_exchange(tmp_path):
    mp.spawn(_bad_world_worker, args=(3, _free_port(), str(tmp_path)), nprocs=3, join=True)
    for r in range(3):
        assert "power of two" in open(tmp_path / f"rank{r}.txt").read()


def test_single_rank_without_a_process_group():
    assert not dist.is_initialized()
    field, log_h, width, log_blowup, p2w, fri = case = CASES["bb_seeded_fri"]
    ops = OracleShardOps(field, 42, log_blowup, p2w)
    res = S.commit_sharded(ops._t(_trace(field, log_h, width, 7)), width, ops, fri=fri)
    lde, layers, root, proof, alpha = _single(case)
    assert np.array_equal(res.root, root) and res.block.shape == lde.shape
    row, sibs = res.open(5)
    rows_ref, sibs_ref = oracle.mmcs_open(layers, [lde], 5)
    assert np.array_equal(row, rows_ref[0]) and all(np.array_equal(a, b) for a, b in zip(sibs, sibs_ref))
    _same_fri(res.fri, proof)
