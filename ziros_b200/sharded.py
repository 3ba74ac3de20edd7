"""One PCS commitment of a trace whose columns are spread over the ranks of a
torch.distributed process group (one process per GPU).

The reference commits a trace on one device: TwoAdicFriPcs::commit
(zkf-backends/src/plonky3.rs:68) is the coset LDE (zkf-metal/src/ntt/p3_adapter.rs:426-459
with p3-dft's coset_lde_batch), rows bit-reversed (zkf-backends/src/wrapping/
stark_to_groth16.rs:2313-2346), then the Poseidon2 MMCS of the result
(vendor/p3-merkle-tree-gpu/src/merkle_tree.rs:84-151).  The LDE is independent per
column; the leaf hash needs whole rows; and with a power-of-two number of ranks G the
tree over the 2^k LDE rows is G subtrees over contiguous row blocks under log2(G) top
levels.  So, for G ranks:

 1. rank r holds columns [c_r, c_{r+1}) of the n x W trace and extends them to
    b*n x W_r (rows bit-reversed);
 2. one all-to-all: row block q (m = b*n / G rows) of every rank's columns goes to
    rank q;
 3. rank q sets the G column blocks side by side: rows [q*m, (q+1)*m) of the LDE a
    single device computes;
 4. rank q commits its block: the subtree whose leaves are exactly those rows;
 5. an all-gather of the G subtree roots; every rank compresses the top log2(G)
    levels and holds the root, equal to the single-device root;
 6. with FRI: alpha (given, or sampled from a transcript that observed the root), the
    alpha-reduction of each rank's rows, an all-gather of the reduced codeword (16 bytes
    per LDE row), and the FRI commit phase on every rank (same inputs, same proof).

Openings are collective: the rank that owns the row answers from its subtree, the top
siblings come from the gathered roots, and the answer is broadcast.  The all-to-all
(and the all-gather of the reduced codeword) are the only data-path collectives.

The per-rank compute is `CudaShardOps` (this process's GPU, through the C ABI).  Any
object with the same methods can stand in for it, which is how the exchange logic is
tested on CPU ranks.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from . import accel as A
from .accel import BABYBEAR


def column_ranges(width: int, world: int) -> List[Tuple[int, int]]:
    """Columns [c0, c1) of each rank: as even as possible, the first ranks one wider."""
    base, extra = divmod(width, world)
    out, c = [], 0
    for r in range(world):
        w = base + (1 if r < extra else 0)
        out.append((c, c + w))
        c += w
    return out


@dataclass
class FriArgs:
    """FRI of the alpha-reduced LDE (TwoAdicFriPcs open without the (x - z) quotient):
    seeded challenges with a given alpha, or transcript=True (alpha, betas and query
    indices from a DuplexChallenger that first observes the trace root)."""
    log_final: int
    num_queries: int
    alpha: Optional[Sequence[int]] = None
    challenge_seed: int = 0
    query_seed: int = 0
    transcript: bool = False


class CudaShardOps:
    """Per-rank compute of the sharded commitment on this process's GPU."""

    def __init__(self, field: int, seed: int, log_blowup: int, p2_width: int = 16, device=None):
        self.field, self.seed, self.log_blowup = field, seed, log_blowup
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("CudaShardOps runs on a CUDA device")
        self.dtype = torch.int32 if field == BABYBEAR else torch.int64
        self.dft = A.CudaDft(field)
        self.mmcs = A.CudaMerkleTreeMmcs(field, seed, p2_width)
        self.digest_elems = self.mmcs.digest_elems

    def empty(self, rows: int, cols: int, ext4: bool = False) -> torch.Tensor:
        return torch.empty((rows, cols), dtype=torch.int32 if ext4 else self.dtype, device=self.device)

    def lde(self, cols: torch.Tensor) -> torch.Tensor:
        out = self.empty(cols.shape[0] << self.log_blowup, cols.shape[1])
        self.dft.coset_lde_batch_dev(cols, self.log_blowup, out, bit_reverse_rows=True)
        return out

    def commit(self, block: torch.Tensor):
        return self.mmcs.commit_dev([block])

    def commit_reduce(self, block: torch.Tensor, alpha):
        """The block's subtree and its rows' alpha-reduction in one pass (BabyBear, width 16)."""
        if self.field != BABYBEAR or self.digest_elems != 8:
            return None
        seg = self.empty(block.shape[0], 4, ext4=True)
        root, tree = self.mmcs.commit_reduce_dev(block, alpha, seg)
        return root, tree, seg

    def open(self, tree, index: int) -> Tuple[np.ndarray, List[np.ndarray]]:
        rows, sibs = self.mmcs.open_batch(index, tree)
        return rows[0], sibs

    def compress(self, left: np.ndarray, right: np.ndarray) -> np.ndarray:
        return self.mmcs.compress(left, right)

    def challenger(self) -> A.Challenger:
        return A.Challenger(self.field, self.seed)

    def combine(self, block: torch.Tensor, alpha) -> torch.Tensor:
        out = self.empty(block.shape[0], 4, ext4=True)
        A.combine_columns_dev(block, alpha, out)
        return out

    def fri(self, codeword: torch.Tensor, args: FriArgs, challenger=None):
        prover = A.CudaFriProver(self.seed, args.log_final, args.num_queries, args.challenge_seed,
                                 args.query_seed)
        return prover.commit_dev(codeword, challenger)


def _group_shape(group) -> Tuple[int, int]:
    """(world size, rank); without an initialised process group, one rank."""
    if not dist.is_initialized():
        if group is not None:
            raise ValueError("a process group was given but torch.distributed is not initialised")
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def _staged(t: torch.Tensor, group) -> bool:
    """gloo moves host tensors only: device tensors cross it through host memory."""
    return t.is_cuda and dist.get_backend(group) == "gloo"


def _all_to_all(send: torch.Tensor, send_splits: List[int], recv_splits: List[int], group) -> torch.Tensor:
    if _group_shape(group)[0] == 1:
        return send
    recv = torch.empty(sum(recv_splits), dtype=send.dtype, device=send.device)
    if _staged(send, group):
        host = torch.empty(sum(recv_splits), dtype=send.dtype)
        dist.all_to_all_single(host, send.cpu(), recv_splits, send_splits, group=group)
        recv.copy_(host)
    else:
        dist.all_to_all_single(recv, send, recv_splits, send_splits, group=group)
    return recv


def _all_gather(t: torch.Tensor, group) -> torch.Tensor:
    """Concatenation over ranks (rank order) of equally shaped tensors."""
    world = _group_shape(group)[0]
    if world == 1:
        return t
    if _staged(t, group):
        parts = [torch.empty_like(t, device="cpu") for _ in range(world)]
        dist.all_gather(parts, t.cpu(), group=group)
        return torch.cat(parts).to(t.device)
    if t.is_cuda:
        out = torch.empty((world * t.shape[0],) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        dist.all_gather_into_tensor(out, t.contiguous(), group=group)
        return out
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return torch.cat(parts)


class ShardedCommitment:
    """Result of commit_sharded on one rank: the root (same on every rank), this rank's
    row block of the LDE and its subtree, the top levels, and the FRI proof if asked."""

    def __init__(self, root, log_n: int, width: int, block, tree, top, rank: int, world: int, group, ops,
                 fri=None, alpha=None):
        self.root = root
        self.log_n = log_n            # log2 of the LDE height
        self.width = width
        self.block = block            # rows [rank*m, (rank+1)*m) of the LDE, all columns
        self.tree = tree              # this rank's subtree
        self.top = top                # top[l]: the G >> l digests at height log2(m) + l
        self.rank, self.world, self.group, self.ops = rank, world, group, ops
        self.fri = fri
        self.alpha = alpha

    @property
    def rows_per_rank(self) -> int:
        return (1 << self.log_n) // self.world

    def open(self, index: int) -> Tuple[np.ndarray, List[np.ndarray]]:
        """Mmcs::open_batch at an LDE row (collective: every rank calls it with the same
        index and gets the same answer): the row and its log2(b*n) sibling digests."""
        if not 0 <= index < (1 << self.log_n):
            raise IndexError(f"row {index} out of range for height 2^{self.log_n}")
        m = self.rows_per_rank
        owner = index // m
        payload = [None]
        if self.rank == owner:
            row, sibs = self.ops.open(self.tree, index % m)
            payload = [(np.asarray(row), [np.asarray(s) for s in sibs])]
        if self.world > 1:
            src = owner if self.group is None else dist.get_global_rank(self.group, owner)
            dist.broadcast_object_list(payload, src=src, group=self.group)
        row, sibs = payload[0]
        sibs = list(sibs) + [self.top[l][(owner >> l) ^ 1].copy() for l in range(len(self.top) - 1)]
        return row, sibs


def commit_sharded(cols: torch.Tensor, width: int, ops, group=None,
                   fri: Optional[FriArgs] = None) -> ShardedCommitment:
    """Collective: rank r passes its columns column_ranges(width, G)[r] of the n x W
    trace (n x W_r, row-major, on ops' device).  G must be a power of two no larger than
    the LDE height.  Without an initialised process group it runs as the only rank.
    Returns this rank's ShardedCommitment."""
    world, rank = _group_shape(group)
    if world & (world - 1):
        raise ValueError(f"the number of ranks ({world}) must be a power of two")
    ranges = column_ranges(width, world)
    c0, c1 = ranges[rank]
    n = int(cols.shape[0])
    if cols.dim() != 2 or cols.shape[1] != c1 - c0:
        raise ValueError(f"rank {rank} holds columns [{c0}, {c1}): expected an n x {c1 - c0} tensor")
    if n < 1 or n & (n - 1):
        raise ValueError("trace height must be a power of two")
    log_n = (n.bit_length() - 1) + ops.log_blowup
    big_n = 1 << log_n
    if big_n < world:
        raise ValueError(f"LDE height 2^{log_n} is smaller than the number of ranks")
    m = big_n // world

    # 1. LDE of this rank's columns (bit-reversed rows)
    lde = ops.lde(cols.contiguous()) if c1 > c0 else ops.empty(big_n, 0)
    if world == 1:
        block = lde  # the only rank holds every column and every row
    else:
        # 2. row block q of every rank's columns goes to rank q (row-major blocks are contiguous)
        widths = [b - a for a, b in ranges]
        send = lde.reshape(-1)
        recv = _all_to_all(send, [m * (c1 - c0)] * world, [m * w for w in widths], group)
        del lde, send
        # 3. the G column blocks side by side
        block = ops.empty(m, width)
        off = 0
        for (a, b), w in zip(ranges, widths):
            if w:
                block[:, a:b].copy_(recv[off:off + m * w].view(m, w))
            off += m * w
        del recv
    # 4. this rank's subtree (with seeded FRI, alpha is known now: the leaf hash also
    # reduces the rows)
    seg = None
    fused = None
    if fri is not None and not fri.transcript and fri.alpha is not None and hasattr(ops, "commit_reduce"):
        fused = ops.commit_reduce(block, np.ascontiguousarray(fri.alpha, dtype=np.uint32))
    if fused is not None:
        sub_root, tree, seg = fused
    else:
        sub_root, tree = ops.commit(block)
    # 5. the subtree roots, then the top levels
    d = ops.digest_elems
    roots_t = _all_gather(torch.as_tensor(np.asarray(sub_root).view(np.int32 if ops.dtype == torch.int32
                                                                      else np.int64))
                          .reshape(1, d).to(ops.device), group)
    roots = roots_t.cpu().numpy().view(np.uint32 if ops.dtype == torch.int32 else np.uint64).reshape(world, d)
    top = [roots]
    while top[-1].shape[0] > 1:
        lvl = top[-1]
        top.append(ops.compress(lvl[0::2], lvl[1::2]).reshape(-1, d))
    root = top[-1][0].copy()
    res = ShardedCommitment(root, log_n, width, block, tree, top, rank, world, group, ops)
    if fri is None:
        return res
    # 6. alpha-reduction of this rank's rows, the whole reduced codeword, FRI
    if ops.field != BABYBEAR:
        raise ValueError("the FRI commit phase runs over BabyBear^4")
    ch = None
    if fri.transcript:
        ch = ops.challenger()
        ch.observe(root.astype(np.uint64))
        alpha = ch.sample(4).astype(np.uint32)
    else:
        if fri.alpha is None:
            raise ValueError("seeded FRI needs alpha")
        alpha = np.ascontiguousarray(fri.alpha, dtype=np.uint32)
    if seg is None:
        seg = ops.combine(block, alpha)
    codeword = _all_gather(seg, group)
    res.fri = ops.fri(codeword, fri, ch)
    res.alpha = alpha
    return res
