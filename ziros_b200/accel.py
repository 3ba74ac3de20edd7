"""Host-side mirror of the reference's accelerator types over the C ABI.

Each class keeps the name, argument meaning and error behaviour of the ZirOS
type it stands in for (paths relative to the ZirOS repository root):

  CudaPoseidon2        <- MetalPoseidon2          zkf-metal/src/poseidon2/mod.rs:21-257
  CudaDft              <- MetalDft<F>             zkf-metal/src/ntt/p3_adapter.rs:36-459
  CudaMerkleTreeMmcs   <- MetalMerkleTreeMmcs     zkf-metal/src/merkle.rs:33-138
  CudaFri              <- MetalFri                zkf-metal/src/fri.rs:18-147

``new()`` returns None when no CUDA device is present, as ``MetalX::new()`` does
without a Metal device; batch calls return ``False`` / ``None`` when the library
declines (the caller then takes its CPU path).  Any other failure raises.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N

BABYBEAR = N.FIELD_BABYBEAR
GOLDILOCKS = N.FIELD_GOLDILOCKS
BB_P = 0x78000001
GL_P = 0xFFFFFFFF00000001


def dtype_of(field: int):
    return np.uint32 if field == BABYBEAR else np.uint64


def _ptr(a: np.ndarray) -> C.c_void_p:
    return a.ctypes.data_as(C.c_void_p)


def _torch_ptr_stream(t):
    import torch

    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr()), C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def round_constants(field: int, seed: int, width: int = 16) -> Tuple[np.ndarray, int, int]:
    """flatten_round_constants(seed) (zkf-metal/src/poseidon2/{babybear,goldilocks}.rs)."""
    lib = N.load()
    out = np.zeros(512, dtype=dtype_of(field))
    ne, ni = C.c_uint32(), C.c_uint32()
    if field == BABYBEAR:
        if width != 16:
            raise ValueError("BabyBear Poseidon2 is width 16")
        n = lib.zkb_poseidon2_babybear_round_constants(seed, _ptr(out), out.size, C.byref(ne), C.byref(ni))
    else:
        n = lib.zkb_poseidon2_goldilocks_round_constants(seed, width, _ptr(out), out.size, C.byref(ne),
                                                         C.byref(ni))
    N.check(n)
    return out[:n].copy(), ne.value, ni.value


def _have_device() -> bool:
    return N.device_count() > 0


# --------------------------------------------------------------------- Poseidon2
class CudaPoseidon2:
    """Batch Poseidon2 width-16 permutations (MetalPoseidon2)."""

    @staticmethod
    def new() -> Optional["CudaPoseidon2"]:
        N.load()
        return CudaPoseidon2() if _have_device() else None

    def batch_permute_babybear(self, states: np.ndarray, round_constants: np.ndarray,
                               n_external_rounds: int, n_internal_rounds: int) -> bool:
        """In-place; False when declined (poseidon2/mod.rs:150-257)."""
        return self._permute(BABYBEAR, states, round_constants, n_external_rounds, n_internal_rounds)

    def batch_permute_goldilocks(self, states: np.ndarray, round_constants: np.ndarray,
                                 n_external_rounds: int, n_internal_rounds: int) -> bool:
        """In-place; False when declined (poseidon2/mod.rs:36-148)."""
        return self._permute(GOLDILOCKS, states, round_constants, n_external_rounds, n_internal_rounds)

    def _permute(self, field, states, rc, ne, ni) -> bool:
        dt = dtype_of(field)
        if states.dtype != dt or not states.flags.c_contiguous:
            raise TypeError(f"states must be a contiguous {np.dtype(dt).name} array")
        rc = np.ascontiguousarray(rc, dtype=dt)
        lib = N.load()
        fn = lib.zkb_poseidon2_babybear_permute if field == BABYBEAR else lib.zkb_poseidon2_goldilocks_permute
        try:
            N.check(fn(_ptr(states), states.size, _ptr(rc), rc.size, ne, ni))
        except N.ZkbDeclined:
            return False
        return True

    def batch_permute_dev(self, field: int, states, round_constants: np.ndarray,
                          n_external_rounds: int, n_internal_rounds: int) -> None:
        """Device-resident form on a CUDA torch tensor, on the tensor's current stream."""
        rc = np.ascontiguousarray(round_constants, dtype=dtype_of(field))
        ptr, stream = _torch_ptr_stream(states)
        lib = N.load()
        fn = (lib.zkb_poseidon2_babybear_permute_dev if field == BABYBEAR
              else lib.zkb_poseidon2_goldilocks_permute_dev)
        N.check(fn(ptr, states.numel(), _ptr(rc), rc.size, n_external_rounds, n_internal_rounds, stream))


# --------------------------------------------------------------------------- DFT
class CudaDft:
    """TwoAdicSubgroupDft over a row-major matrix (MetalDft<F>)."""

    def __init__(self, field: int):
        N.load()
        self.field = field

    @staticmethod
    def new(field: int) -> Optional["CudaDft"]:
        N.load()
        return CudaDft(field) if _have_device() else None

    def _mat(self, mat: np.ndarray) -> np.ndarray:
        m = np.ascontiguousarray(mat, dtype=dtype_of(self.field))
        if m.ndim == 1:
            m = m.reshape(-1, 1)
        h = m.shape[0]
        if h == 0 or h & (h - 1):
            raise ValueError("height must be a power of two")
        return m

    def dft_batch(self, mat: np.ndarray) -> np.ndarray:
        m = self._mat(mat).copy()
        N.check(N.load().zkb_dft_batch(self.field, _ptr(m), m.shape[0].bit_length() - 1, m.shape[1], 0))
        return m

    def idft_batch(self, mat: np.ndarray) -> np.ndarray:
        m = self._mat(mat).copy()
        N.check(N.load().zkb_dft_batch(self.field, _ptr(m), m.shape[0].bit_length() - 1, m.shape[1], 1))
        return m

    def coset_lde_batch(self, mat: np.ndarray, added_bits: int, shift: Optional[int] = None,
                        bit_reverse_rows: bool = False) -> np.ndarray:
        """p3 coset_lde_batch (natural order), or the PCS's bit-reversed rows."""
        m = self._mat(mat)
        out = np.zeros((m.shape[0] << added_bits, m.shape[1]), dtype=dtype_of(self.field))
        N.check(N.load().zkb_coset_lde_batch(self.field, _ptr(m), m.shape[0].bit_length() - 1, m.shape[1],
                                             added_bits, shift or 0, int(bit_reverse_rows), _ptr(out)))
        return out

    def coset_lde_batch_dev(self, trace, log_blowup: int, out, shift: Optional[int] = None,
                            bit_reverse_rows: bool = True) -> None:
        """Device form on CUDA torch tensors (trace: h x w, out: (h << log_blowup) x w)."""
        h, w = trace.shape
        tp, stream = _torch_ptr_stream(trace)
        op, _ = _torch_ptr_stream(out)
        if out.shape[0] != h << log_blowup or out.shape[1] != w:
            raise ValueError("output shape mismatch")
        N.check(N.load().zkb_coset_lde_batch_dev(self.field, tp, h.bit_length() - 1, w, log_blowup,
                                                 shift or 0, int(bit_reverse_rows), op, stream))


    def coset_lde_tuned_dev(self, trace, log_blowup: int, out, kmax: int = 0, c_pass: int = 0,
                            c_fused: int = 0) -> None:
        """Device LDE (bit-reversed rows) with explicit kernel shapes (0 = default)."""
        h, w = trace.shape
        tp, stream = _torch_ptr_stream(trace)
        op, _ = _torch_ptr_stream(out)
        if out.shape[0] != h << log_blowup or out.shape[1] != w:
            raise ValueError("output shape mismatch")
        N.check(N.load().zkb_coset_lde_tuned_dev(self.field, tp, h.bit_length() - 1, w, log_blowup, kmax, c_pass,
                                                 c_fused, op, stream))


class CudaNttAccelerator:
    """NttAccelerator (zkf-core/src/acceleration.rs:62-81) as MetalNttAccelerator
    implements it (zkf-metal/src/ntt/mod.rs:13-109): a Goldilocks transform of one
    column, natural order in place.  Each value's low 64 bits are reduced into the
    field (Goldilocks::from_u64 of the first 8 little-endian bytes), the transform runs
    through zkb_dft_batch(GOLDILOCKS, width 1) and the canonical results are written
    back.  forward_ntt is the DFT, inverse_ntt the inverse DFT with the 1/n scale."""

    def __init__(self):
        N.load()

    @staticmethod
    def new() -> Optional["CudaNttAccelerator"]:
        N.load()
        return CudaNttAccelerator() if _have_device() else None

    def name(self) -> str:
        return "cuda-b200-ntt"

    def is_available(self) -> bool:
        return _have_device()

    def max_log_size(self) -> int:
        return 26

    def _run(self, values: list, inverse: int) -> None:
        n = len(values)
        if n == 0 or n & (n - 1):
            raise N.ZkbError(N.ERR_INVALID, "NTT size must be a power of 2")
        if n.bit_length() - 1 > self.max_log_size():
            raise N.ZkbError(N.ERR_INVALID, f"NTT of 2^{n.bit_length() - 1} exceeds max_log_size 2^26")
        v = np.array([(int(x) & 0xFFFFFFFFFFFFFFFF) % GL_P for x in values], dtype=np.uint64)
        N.check(N.load().zkb_dft_batch(GOLDILOCKS, _ptr(v), n.bit_length() - 1, 1, inverse))
        values[:] = [int(x) for x in v]

    def forward_ntt(self, values: list) -> None:
        self._run(values, 0)

    def inverse_ntt(self, values: list) -> None:
        self._run(values, 1)


# -------------------------------------------------------------------------- MMCS
class Tree:
    """Prover data of a commitment (p3 MerkleTree): digest layers stay on the device."""

    def __init__(self, handle: C.c_void_p, field: int, shapes: Sequence[Tuple[int, int]], owner=None):
        self._h = handle
        self.field = field
        self.heights = [int(s[0]) for s in shapes]
        self.widths = [int(s[1]) for s in shapes]
        self._owner = owner  # a borrowed tree keeps the object that owns it alive

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h and getattr(self, "_owner", None) is None:
            try:
                N.load().zkb_tree_free(h)
            except Exception:  # interpreter shutdown: module state already torn down
                pass

    @property
    def digest_elems(self) -> int:
        return N.load().zkb_tree_digest_elems(self._h)

    def num_layers(self) -> int:
        return N.load().zkb_tree_num_layers(self._h)

    def layer(self, i: int) -> np.ndarray:
        lib = N.load()
        n = lib.zkb_tree_layer_len(self._h, i)
        N.check(n if n < 0 else 0)
        out = np.zeros((n, self.digest_elems), dtype=dtype_of(self.field))
        N.check(lib.zkb_tree_copy_layer(self._h, i, _ptr(out)))
        return out

    def digest_layers(self) -> List[np.ndarray]:
        return [self.layer(i) for i in range(self.num_layers())]

    def root(self) -> np.ndarray:
        return self.layer(self.num_layers() - 1)[0]


class CudaMerkleTreeMmcs:
    """Poseidon2 MMCS (MetalMerkleTreeMmcs / p3 MerkleTreeMmcs) with device-resident layers."""

    def __init__(self, field: int, seed: int, width: int = 16):
        N.load()
        self.field = field
        self.hasher = N.Hasher(field, width, seed)
        self.digest_elems = 8 if width == 16 else 4

    def commit(self, mats: Sequence[np.ndarray]) -> Tuple[np.ndarray, Tree]:
        """Mmcs::commit -> (root, prover data)."""
        dt = dtype_of(self.field)
        mats = [np.ascontiguousarray(m, dtype=dt) for m in mats]
        descs = (N.Matrix * len(mats))(*[N.Matrix(m.ctypes.data, m.shape[0], m.shape[1]) for m in mats])
        root = np.zeros(self.digest_elems, dtype=dt)
        handle = C.c_void_p()
        N.check(N.load().zkb_mmcs_commit(C.byref(self.hasher), descs, len(mats), _ptr(root), C.byref(handle)))
        return root, Tree(handle, self.field, [m.shape for m in mats])

    def commit_dev(self, mats) -> Tuple[np.ndarray, Tree]:
        """Commit CUDA torch tensors in place; they must outlive the returned tree."""
        import torch

        descs = (N.Matrix * len(mats))(*[N.Matrix(m.data_ptr(), m.shape[0], m.shape[1]) for m in mats])
        root = np.zeros(self.digest_elems, dtype=dtype_of(self.field))
        handle = C.c_void_p()
        stream = C.c_void_p(torch.cuda.current_stream(mats[0].device).cuda_stream)
        N.check(N.load().zkb_mmcs_commit_dev(C.byref(self.hasher), descs, len(mats), _ptr(root),
                                             C.byref(handle), stream))
        t = Tree(handle, self.field, [tuple(m.shape) for m in mats])
        t._keepalive = list(mats)
        return root, t

    def verify_batch(self, root, shapes: Sequence[Tuple[int, int]], index: int, rows: Sequence[np.ndarray],
                     siblings: Sequence[np.ndarray]) -> bool:
        """Mmcs::verify_batch: True when the opening reproduces the root (host-side)."""
        dt = dtype_of(self.field)
        r = np.ascontiguousarray(root, dtype=dt)
        hs = np.array([s[0] for s in shapes], np.uint64)
        ws = np.array([s[1] for s in shapes], np.uint64)
        cat = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=dt).reshape(-1) for x in rows]), dtype=dt)
        sib = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=dt).reshape(-1) for x in siblings])
                                   if len(siblings) else np.zeros(0, dt), dtype=dt)
        rc = N.load().zkb_mmcs_verify_batch(C.byref(self.hasher), _ptr(r), _ptr(hs), _ptr(ws), len(shapes), index,
                                            _ptr(cat), _ptr(sib), len(siblings))
        if rc == N.ERR_INVALID:
            return False
        N.check(rc)
        return True

    def commit_reduce_dev(self, mat, alpha, codeword) -> Tuple[np.ndarray, Tree]:
        """Commit one CUDA int32 matrix (BabyBear, width-16 hasher) and write its rows'
        alpha-reduction into `codeword` (rows x 4 int32 CUDA tensor) in the same pass."""
        import torch

        if codeword.shape != (mat.shape[0], 4):
            raise ValueError("codeword must be rows x 4")
        desc = N.Matrix(mat.data_ptr(), mat.shape[0], mat.shape[1])
        a = np.ascontiguousarray(alpha, dtype=np.uint32)
        root = np.zeros(self.digest_elems, dtype=dtype_of(self.field))
        handle = C.c_void_p()
        stream = C.c_void_p(torch.cuda.current_stream(mat.device).cuda_stream)
        N.check(N.load().zkb_mmcs_commit_reduce_dev(C.byref(self.hasher), C.byref(desc), _ptr(a), _ptr(root),
                                                    C.byref(handle), C.c_void_p(codeword.data_ptr()), stream))
        t = Tree(handle, self.field, [tuple(mat.shape)])
        t._keepalive = [mat]
        return root, t

    def compress(self, left, right) -> np.ndarray:
        """TruncatedPermutation of digest pairs (host): left, right (n, OUT) -> (n, OUT)."""
        dt = dtype_of(self.field)
        lt = np.ascontiguousarray(left, dtype=dt).reshape(-1, self.digest_elems)
        rt = np.ascontiguousarray(right, dtype=dt).reshape(-1, self.digest_elems)
        if lt.shape != rt.shape:
            raise ValueError("left and right hold different numbers of digests")
        out = np.zeros_like(lt)
        N.check(N.load().zkb_mmcs_compress(C.byref(self.hasher), _ptr(lt), _ptr(rt), lt.shape[0], _ptr(out)))
        return out

    def open_batch(self, index: int, tree: Tree) -> Tuple[List[np.ndarray], List[np.ndarray]]:
        """Mmcs::open_batch -> (rows per matrix, sibling digests)."""
        dt = dtype_of(self.field)
        total_w = sum(tree.widths)
        log_max = (max(tree.heights) - 1).bit_length()
        rows = np.zeros(max(total_w, 1), dtype=dt)
        sib = np.zeros(max(log_max * self.digest_elems, 1), dtype=dt)
        N.check(N.load().zkb_mmcs_open_batch(tree._h, index, _ptr(rows), rows.size, _ptr(sib), sib.size))
        out, off = [], 0
        for w in tree.widths:
            out.append(rows[off:off + w].copy())
            off += w
        return out, [sib[i * self.digest_elems:(i + 1) * self.digest_elems].copy() for i in range(log_max)]


# ----------------------------------------------------------------------- PCS
class CudaTwoAdicPcs:
    """TwoAdicFriPcs::commit for a trace matrix (Pcs at zkf-backends/src/plonky3.rs:68):
    coset LDE by 2^log_blowup, bit-reversed rows, Poseidon2 MMCS commit.  The LDE stays
    on the device as the tree's leaf matrix."""

    def __init__(self, field: int, seed: int, log_blowup: int, width: int = 16):
        self.mmcs = CudaMerkleTreeMmcs(field, seed, width)
        self.field = field
        self.log_blowup = log_blowup

    def commit(self, trace: np.ndarray) -> Tuple[np.ndarray, Tree]:
        t = np.ascontiguousarray(trace, dtype=dtype_of(self.field))
        h, w = t.shape
        root = np.zeros(self.mmcs.digest_elems, dtype=dtype_of(self.field))
        handle = C.c_void_p()
        N.check(N.load().zkb_pcs_commit(C.byref(self.mmcs.hasher), _ptr(t), h.bit_length() - 1, w,
                                        self.log_blowup, _ptr(root), C.byref(handle)))
        return root, Tree(handle, self.field, [(h << self.log_blowup, w)])

    def commit_ptr(self, host_ptr: int, height: int, width: int, want_tree: bool = True,
                   root: Optional[np.ndarray] = None):
        """Host-pointer form for caller-managed (e.g. pinned) buffers."""
        root = np.zeros(self.mmcs.digest_elems, dtype=dtype_of(self.field)) if root is None else root
        handle = C.c_void_p()
        N.check(N.load().zkb_pcs_commit(C.byref(self.mmcs.hasher), C.c_void_p(host_ptr),
                                        height.bit_length() - 1, width, self.log_blowup, _ptr(root),
                                        C.byref(handle) if want_tree else None))
        tree = Tree(handle, self.field, [(height << self.log_blowup, width)]) \
            if want_tree else None
        return root, tree

    def commit_dev(self, trace, want_tree: bool = True, root: Optional[np.ndarray] = None):
        """Device form on a CUDA torch tensor (h x w), on the tensor's current stream."""
        h, w = trace.shape
        ptr, stream = _torch_ptr_stream(trace)
        root = np.zeros(self.mmcs.digest_elems, dtype=dtype_of(self.field)) if root is None else root
        handle = C.c_void_p()
        N.check(N.load().zkb_pcs_commit_dev(C.byref(self.mmcs.hasher), ptr, h.bit_length() - 1, w,
                                            self.log_blowup, _ptr(root),
                                            C.byref(handle) if want_tree else None, stream))
        tree = Tree(handle, self.field, [(h << self.log_blowup, w)]) \
            if want_tree else None
        return root, tree


    # -- commit + FRI job (BabyBear) ------------------------------------------------
    def _fri_call(self, dev: bool, ptr, stream, h: int, w: int, alpha, log_final: int, num_queries: int,
                  challenge_seed: int, query_seed: int, want_tree: bool, root, transcript: bool = False):
        a = np.ascontiguousarray(alpha if alpha is not None else np.zeros(4), dtype=np.uint32)
        log_n = (h.bit_length() - 1) + self.log_blowup
        prm = N.FriParams(log_n, log_final, challenge_seed, num_queries, query_seed, int(transcript))
        root = np.zeros(8, np.uint32) if root is None else root
        th, fh = C.c_void_p(), C.c_void_p()
        args = [C.byref(self.mmcs.hasher), ptr, h.bit_length() - 1, w, self.log_blowup, _ptr(a), C.byref(prm),
                _ptr(root), C.byref(th) if want_tree else None, C.byref(fh)]
        lib = N.load()
        if dev:
            N.check(lib.zkb_pcs_commit_fri_dev(*args, stream))
        else:
            N.check(lib.zkb_pcs_commit_fri(*args))
        tree = Tree(th, self.field, [(h << self.log_blowup, w)]) if want_tree else None
        return root, tree, FriProof(fh, prm)

    def commit_fri(self, trace: np.ndarray, alpha, log_final: int, num_queries: int, challenge_seed: int = 0,
                   query_seed: int = 0, want_tree: bool = True, transcript: bool = False):
        """Commit the trace, reduce its LDE columns with alpha, run the FRI commit phase:
        returns (root, tree, FriProof).  transcript=True draws alpha, the betas and the
        query indices from the Fiat-Shamir transcript (alpha and the seeds are ignored)."""
        t = np.ascontiguousarray(trace, dtype=np.uint32)
        return self._fri_call(False, _ptr(t), None, t.shape[0], t.shape[1], alpha, log_final, num_queries,
                              challenge_seed, query_seed, want_tree, None, transcript)

    def commit_fri_ptr(self, host_ptr: int, height: int, width: int, alpha, log_final: int, num_queries: int,
                       challenge_seed: int = 0, query_seed: int = 0, want_tree: bool = False, root=None,
                       transcript: bool = False):
        return self._fri_call(False, C.c_void_p(host_ptr), None, height, width, alpha, log_final, num_queries,
                              challenge_seed, query_seed, want_tree, root, transcript)

    def commit_fri_dev(self, trace, alpha, log_final: int, num_queries: int, challenge_seed: int = 0,
                       query_seed: int = 0, want_tree: bool = False, root=None, transcript: bool = False):
        ptr, stream = _torch_ptr_stream(trace)
        return self._fri_call(True, ptr, stream, trace.shape[0], trace.shape[1], alpha, log_final, num_queries,
                              challenge_seed, query_seed, want_tree, root, transcript)


# --------------------------------------------------------------------------- FRI
class CudaFri:
    """FRI folding (MetalFri / FriAccelerator)."""

    @staticmethod
    def new() -> Optional["CudaFri"]:
        N.load()
        return CudaFri() if _have_device() else None

    def _fold(self, field, evals, alpha, inv_twiddles):
        dt = dtype_of(field)
        e = np.ascontiguousarray(evals, dtype=dt)
        if e.size % 2:
            return None
        t = None if inv_twiddles is None else np.ascontiguousarray(inv_twiddles, dtype=dt)
        if t is not None and t.size != e.size // 2:
            return None
        out = np.zeros(e.size // 2, dtype=dt)
        lib = N.load()
        fn = lib.zkb_fri_fold_goldilocks if field == GOLDILOCKS else lib.zkb_fri_fold_babybear
        try:
            N.check(fn(_ptr(e), e.size, alpha, None if t is None else _ptr(t), _ptr(out)))
        except N.ZkbDeclined:
            return None
        return out

    def fold_goldilocks(self, evals, alpha: int, inv_twiddles=None) -> Optional[np.ndarray]:
        return self._fold(GOLDILOCKS, evals, alpha, inv_twiddles)

    def fold_babybear(self, evals, alpha: int, inv_twiddles=None) -> Optional[np.ndarray]:
        return self._fold(BABYBEAR, evals, alpha, inv_twiddles)

    def fold_babybear_ext4(self, evals: np.ndarray, beta) -> np.ndarray:
        """p3 fold_matrix over BabyBear^4; evals: (2n, 4) u32 -> (n, 4)."""
        e = np.ascontiguousarray(evals, dtype=np.uint32).reshape(-1, 4)
        b = np.ascontiguousarray(beta, dtype=np.uint32)
        out = np.zeros((e.shape[0] // 2, 4), dtype=np.uint32)
        N.check(N.load().zkb_fri_fold_babybear_ext4(_ptr(e), out.shape[0], _ptr(b), _ptr(out)))
        return out


class FriProof:
    """Result of the FRI commit phase: per-round roots and betas, final codeword and
    query openings (all on the host)."""

    def __init__(self, handle: C.c_void_p, params: "N.FriParams"):
        lib = N.load()
        self._h = handle
        self.log_n, self.log_final = params.log_n, params.log_final
        self.rounds = lib.zkb_fri_num_rounds(handle)
        if self.rounds != self.log_n - self.log_final:
            raise N.ZkbError(f"FRI proof has {self.rounds} rounds, expected {self.log_n - self.log_final}")
        self.roots = np.zeros((self.rounds, 8), np.uint32)
        self.betas = np.zeros((self.rounds, 4), np.uint32)
        N.check(lib.zkb_fri_commitments(handle, _ptr(self.roots), _ptr(self.betas)))
        self.final = np.zeros((1 << self.log_final, 4), np.uint32)
        N.check(lib.zkb_fri_final_codeword(handle, _ptr(self.final)))
        self.alpha = np.zeros(4, np.uint32)  # the column-reduction alpha of a commit+FRI job
        N.check(lib.zkb_fri_alpha(handle, _ptr(self.alpha)))
        nq = params.num_queries
        spq = lib.zkb_fri_siblings_per_query(handle)
        self.query_indices = np.zeros(nq, np.uint64)
        self.query_rows = np.zeros((nq, self.rounds, 8), np.uint32)
        self.query_siblings = np.zeros((nq, max(spq, 0)), np.uint32)
        if nq:
            N.check(lib.zkb_fri_query_openings(handle, _ptr(self.query_indices), _ptr(self.query_rows),
                                               _ptr(self.query_siblings)))

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                N.load().zkb_fri_proof_free(h)
            except Exception:  # interpreter shutdown: module state already torn down
                pass

    def siblings(self, q: int, r: int) -> np.ndarray:
        """Sibling digests of query q in round r: (log_n - r - 1, 8)."""
        off = sum(self.log_n - k - 1 for k in range(r)) * 8
        depth = self.log_n - r - 1
        return self.query_siblings[q, off:off + depth * 8].reshape(depth, 8)


class CudaFriProver:
    """FRI commit phase over BabyBear^4 (p3 prove_fri's commit phase and query answers,
    as TwoAdicFriPcs runs them), with seeded challenges or, with transcript=True,
    challenges drawn from a fresh DuplexChallenger."""

    def __init__(self, seed: int, log_final: int, num_queries: int, challenge_seed: int = 0,
                 query_seed: int = 0, transcript: bool = False):
        N.load()
        self.hasher = N.Hasher(BABYBEAR, 16, seed)
        self.log_final = log_final
        self.num_queries = num_queries
        self.challenge_seed = challenge_seed
        self.query_seed = query_seed
        self.transcript = transcript

    def _params(self, log_n: int) -> "N.FriParams":
        return N.FriParams(log_n, self.log_final, self.challenge_seed, self.num_queries, self.query_seed,
                           int(self.transcript))

    def commit(self, codeword: np.ndarray) -> FriProof:
        cw = np.ascontiguousarray(codeword, dtype=np.uint32).reshape(-1, 4)
        log_n = cw.shape[0].bit_length() - 1
        prm = self._params(log_n)
        h = C.c_void_p()
        N.check(N.load().zkb_fri_commit_babybear_ext4(C.byref(self.hasher), C.byref(prm), _ptr(cw), C.byref(h)))
        return FriProof(h, prm)

    def commit_dev(self, codeword, challenger: Optional["Challenger"] = None) -> FriProof:
        """codeword: CUDA tensor of 2^log_n x 4 int32 (extension coefficients).  With a
        challenger, the challenges come from it (its state advanced by the call), as when
        one transcript runs from the trace commitment into FRI."""
        log_n = codeword.shape[0].bit_length() - 1
        prm = self._params(log_n)
        ptr, stream = _torch_ptr_stream(codeword)
        h = C.c_void_p()
        lib = N.load()
        if challenger is None:
            N.check(lib.zkb_fri_commit_babybear_ext4_dev(C.byref(self.hasher), C.byref(prm), ptr, C.byref(h),
                                                         stream))
        else:
            prm.transcript = 1
            N.check(lib.zkb_fri_commit_babybear_ext4_challenger_dev(C.byref(self.hasher), C.byref(prm), ptr,
                                                                    challenger._h, C.byref(h), stream))
        return FriProof(h, prm)


def combine_columns_dev(lde, alpha, out) -> None:
    """out[i] = sum_j alpha^j lde[i][j] over BabyBear^4 (CUDA tensors: rows x w, rows x 4)."""
    a = np.ascontiguousarray(alpha, dtype=np.uint32)
    lp, stream = _torch_ptr_stream(lde)
    op, _ = _torch_ptr_stream(out)
    N.check(N.load().zkb_combine_columns_babybear_ext4_dev(lp, lde.shape[0], lde.shape[1], _ptr(a), op, stream))


class CommitEngine:
    """Continuous-batching commit engine (zkb_engine_*): jobs are submitted without
    blocking, admitted by free HBM and slot, and overlap on the device."""

    POLICIES = {"fifo": N.ADMIT_FIFO, "smallest": N.ADMIT_SMALLEST}

    def __init__(self, slots: int = 2, hbm_budget: int = 0, policy: str = "fifo"):
        """policy "fifo" (default): oldest fitting job first; "smallest": fewest cells
        first.  Under both a job passed over ADMIT_MAX_BYPASS times goes next."""
        lib = N.load()
        self._h = C.c_void_p()
        if policy not in self.POLICIES:
            raise ValueError(f"unknown admission policy {policy!r}")
        cfg = N.EngineConfig(slots, hbm_budget, self.POLICIES[policy])
        N.check(lib.zkb_engine_create(C.byref(cfg), C.byref(self._h)))
        self._keep = {}

    def submit(self, trace, field: int = BABYBEAR, seed: int = 42, log_blowup: int = 1, p2_width: int = 16,
               fri: Optional[dict] = None, host_ptr: Optional[int] = None, shape=None) -> int:
        """trace: host array (kept alive until the job is waited on), or host_ptr + shape."""
        if host_ptr is None:
            t = np.ascontiguousarray(trace, dtype=dtype_of(field))
            ptr, (h, w) = t.ctypes.data, t.shape
        else:
            t, ptr, (h, w) = trace, host_ptr, shape
        d = N.JobDesc()
        d.hasher = N.Hasher(field, p2_width, seed)
        d.trace = ptr
        d.log_h, d.width, d.log_blowup = h.bit_length() - 1, w, log_blowup
        if fri:
            d.with_fri = 1
            d.alpha[:] = [int(x) for x in fri.get("alpha", [0, 0, 0, 0])]
            d.fri = N.FriParams(0, fri["log_final"], fri.get("challenge_seed", 0), fri["num_queries"],
                                fri.get("query_seed", 0), int(fri.get("transcript", False)))
        jid = C.c_uint64()
        N.check(N.load().zkb_engine_submit(self._h, C.byref(d), C.byref(jid)))
        self._keep[jid.value] = (t, d)
        return jid.value

    def wait(self, job_id: int):
        """-> (root, FriProof or None, {queue_ms, run_ms, latency_ms})"""
        res = N.JobResult()
        fh = C.c_void_p()
        rc = N.load().zkb_engine_wait(self._h, job_id, C.byref(res), C.byref(fh))
        _, d = self._keep.pop(job_id)
        N.check(rc)
        field = d.hasher.field
        out = 8 if d.hasher.width == 16 else 4
        raw = np.array(res.root[:], dtype=np.uint32)
        root = raw[:out] if field == BABYBEAR else raw.view(np.uint64)[:out]
        pf = None
        if fh:
            prm = N.FriParams(d.log_h + d.log_blowup, d.fri.log_final, d.fri.challenge_seed, d.fri.num_queries,
                              d.fri.query_seed, d.fri.transcript)
            pf = FriProof(fh, prm)
        return root, pf, {"queue_ms": res.queue_ms, "run_ms": res.run_ms, "latency_ms": res.latency_ms}

    def cancel(self, job_id: int) -> bool:
        """Cancels a queued job (its wait then raises with ERR_CANCELLED); False when it
        has already started."""
        rc = N.load().zkb_engine_cancel(self._h, job_id)
        if rc == N.DECLINED:
            return False
        N.check(rc)
        return True

    def stats(self) -> dict:
        st = N.EngineStats()
        N.check(N.load().zkb_engine_stats(self._h, C.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in N.EngineStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            N.load().zkb_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ------------------------------------------------------------------ polynomial ops
class CudaPolyOps:
    """PolyOpsAccelerator (MetalPolyOps, zkf-metal/src/poly.rs): Goldilocks batch
    evaluation, coset evaluation and the opening quotient."""

    @staticmethod
    def new() -> Optional["CudaPolyOps"]:
        N.load()
        return CudaPolyOps() if _have_device() else None

    @staticmethod
    def _u64(a) -> np.ndarray:
        return np.ascontiguousarray(a, dtype=np.uint64)

    def batch_eval_goldilocks(self, coeffs, points) -> np.ndarray:
        c, p = self._u64(coeffs), self._u64(points)
        out = np.zeros(p.size, np.uint64)
        N.check(N.load().zkb_poly_eval_goldilocks(_ptr(c), c.size, _ptr(p), p.size, _ptr(out)))
        return out

    def coset_eval_goldilocks(self, coeffs, shift: int, log_n: int) -> np.ndarray:
        c = self._u64(coeffs)
        if c.size != 1 << log_n:
            raise ValueError("need 2^log_n coefficients")
        out = np.zeros(c.size, np.uint64)
        N.check(N.load().zkb_poly_coset_eval_goldilocks(_ptr(c), log_n, shift, _ptr(out)))
        return out

    def quotient_goldilocks(self, evals, z: int, f_z: int) -> np.ndarray:
        e = self._u64(evals)
        n = e.size
        if n == 0 or n & (n - 1):
            raise ValueError("need a power-of-two number of evaluations")
        out = np.zeros(n, np.uint64)
        N.check(N.load().zkb_poly_quotient_goldilocks(_ptr(e), n.bit_length() - 1, z, f_z, _ptr(out)))
        return out


# ------------------------------------------------------------------ runtime driver
class ProverRuntime:
    """GpuDispatchDriver for the prover runtime's nodes (zkb_rt_*): device buffer slots
    and Ntt / Lde / PoseidonBatch / Merkle / FriFold / FriQueryOpen nodes that depend on
    earlier nodes.  execute() returns None, or the id of the node the device path
    declined (the reference's FallbackSignal: run that node and the rest on the CPU)."""

    NTT, LDE, POSEIDON_BATCH, MERKLE, FRI_FOLD, FRI_QUERY_OPEN = 1, 2, 3, 4, 5, 6

    def __init__(self):
        self._h = C.c_void_p()
        N.check(N.load().zkb_rt_create(C.byref(self._h)))

    def buffer(self, nbytes: int) -> int:
        slot = C.c_int()
        N.check(N.load().zkb_rt_buffer(self._h, nbytes, C.byref(slot)))
        return slot.value

    def write(self, slot: int, array: np.ndarray) -> None:
        a = np.ascontiguousarray(array)
        N.check(N.load().zkb_rt_write(self._h, slot, _ptr(a), a.nbytes))

    def read(self, slot: int, shape, dtype) -> np.ndarray:
        out = np.zeros(shape, dtype=dtype)
        N.check(N.load().zkb_rt_read(self._h, slot, _ptr(out), out.nbytes))
        return out

    def add(self, kind: int, field: int = BABYBEAR, deps=(), log_n: int = 0, width: int = 0, log_blowup: int = 0,
            inverse: bool = False, count: int = 0, in_slot: int = -1, out_slot: int = -1, seed: int = 42,
            hasher_width: int = 16, ext4: bool = False, beta=(0, 0, 0, 0), tree_node: int = -1) -> int:
        nd = N.RtNode(kind, field, log_n, width, log_blowup, int(inverse), count, in_slot, out_slot, seed,
                      hasher_width, int(ext4), (C.c_uint32 * 4)(*[int(b) for b in beta]), tree_node)
        d = np.ascontiguousarray(np.array(deps, dtype=np.int32))
        nid = C.c_int()
        N.check(N.load().zkb_rt_add(self._h, C.byref(nd), _ptr(d) if d.size else None, d.size, C.byref(nid)))
        return nid.value

    def execute(self) -> Optional[int]:
        fb = C.c_int(-1)
        rc = N.load().zkb_rt_execute(self._h, None, C.byref(fb))
        if rc == N.DECLINED:
            return fb.value
        N.check(rc)
        return None

    def node_ms(self, node: int) -> float:
        ms = C.c_float()
        N.check(N.load().zkb_rt_node_ms(self._h, node, C.byref(ms)))
        return ms.value

    def tree(self, node: int, height: int, width: int, field: int = BABYBEAR) -> Tree:
        """The tree of an executed Merkle node (borrowed from the runtime)."""
        t = C.c_void_p()
        N.check(N.load().zkb_rt_tree(self._h, node, C.byref(t)))
        return Tree(t, field, [(height, width)], owner=self)

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                N.load().zkb_rt_free(h)
            except Exception:  # interpreter shutdown
                pass


# ------------------------------------------------------------------ transcript
class Challenger:
    """p3 DuplexChallenger<F, Poseidon2<16>, 16, 8> (zkb_challenger_*): observe canonical
    field elements, sample elements or low bits.  Host-side; needs no device."""

    def __init__(self, field: int = BABYBEAR, seed: int = 42):
        self._h = C.c_void_p()
        N.check(N.load().zkb_challenger_create(C.byref(N.Hasher(field, 16, seed)), C.byref(self._h)))

    def observe(self, values) -> None:
        v = np.ascontiguousarray(np.atleast_1d(values), dtype=np.uint64)
        N.check(N.load().zkb_challenger_observe(self._h, _ptr(v), v.size))

    def sample(self, n: int = 1) -> np.ndarray:
        out = np.zeros(n, np.uint64)
        N.check(N.load().zkb_challenger_sample(self._h, _ptr(out), n))
        return out

    def sample_bits(self, bits: int) -> int:
        out = C.c_uint64()
        N.check(N.load().zkb_challenger_sample_bits(self._h, bits, C.byref(out)))
        return out.value

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                N.load().zkb_challenger_free(h)
            except Exception:  # interpreter shutdown
                pass


# ------------------------------------------------------------------ batched commit
class BatchCommit:
    """Many traces of uneven height and width committed by one plan (zkb_batch_*): one
    device arena, tables built once, kernel shapes autotuned (JSON-lines cache), and one
    CUDA graph per run — of ordinary kernels, or with persistent=True of ONE persistent
    kernel fed by a device work queue (BabyBear, widths that are multiples of 8), whose
    Merkle-level fusion the autotuner also chooses.  Every root equals the trace's plain
    commitment (CudaTwoAdicPcs.commit)."""

    def __init__(self, shapes: Sequence[Tuple[int, int]], field: int = BABYBEAR, seed: int = 42,
                 log_blowup: int = 1, p2_width: int = 16, use_graph: bool = True, branches: int = 0,
                 autotune: bool = True, tune_cache: Optional[str] = None, persistent: bool = False):
        lib = N.load()
        self.field = field
        self.shapes = [(int(h), int(w)) for h, w in shapes]
        for h, w in self.shapes:
            if h <= 0 or h & (h - 1):
                raise ValueError("trace heights must be powers of two")
        self.log_blowup = log_blowup
        self.digest_elems = 8 if p2_width == 16 else 4
        self.hasher = N.Hasher(field, p2_width, seed)
        arr = (N.BatchShape * len(self.shapes))(*[N.BatchShape(h.bit_length() - 1, w) for h, w in self.shapes])
        opt = N.BatchOptions(log_blowup, 2 if persistent else int(use_graph), branches, int(autotune),
                             tune_cache.encode() if tune_cache else None)
        self._h = C.c_void_p()
        N.check(lib.zkb_batch_create(C.byref(self.hasher), arr, len(self.shapes), C.byref(opt), C.byref(self._h)))

    def __len__(self):
        return len(self.shapes)

    def copy_in(self, i: int, trace, stream=None) -> None:
        """trace: a host array, a pinned host torch tensor (asynchronous: keep it alive
        until the stream has passed the copy) or a CUDA torch tensor."""
        lib = N.load()
        h, w = self.shapes[i]
        if hasattr(trace, "is_cuda"):
            if tuple(trace.shape) != (h, w) or trace.element_size() != np.dtype(dtype_of(self.field)).itemsize:
                raise ValueError("trace shape/type mismatch")
            s = stream if stream is not None else _current_stream(trace)
            N.check(lib.zkb_batch_copy_in(self._h, i, C.c_void_p(trace.data_ptr()), int(trace.is_cuda), s))
            return
        a = np.ascontiguousarray(trace, dtype=dtype_of(self.field))
        if a.shape != (h, w):
            raise ValueError("trace shape mismatch")
        # a pageable source is staged before the call returns
        N.check(lib.zkb_batch_copy_in(self._h, i, _ptr(a), 0, stream))

    def run(self, stream=None) -> None:
        N.check(N.load().zkb_batch_run(self._h, stream))

    def run_host(self, traces, stream=None) -> None:
        """One run from host memory, the copies overlapped with the commitment
        (zkb_batch_run_host).  traces: one per shape, host arrays (staged before the call
        returns) or pinned host torch tensors (asynchronous: keep them alive until the
        stream has passed the run)."""
        if len(traces) != len(self.shapes):
            raise ValueError("one trace per shape")
        isz = np.dtype(dtype_of(self.field)).itemsize
        keep, ptrs = [], (C.c_void_p * len(self.shapes))()
        for i, (t, (h, w)) in enumerate(zip(traces, self.shapes)):
            if hasattr(t, "is_cuda"):
                if t.is_cuda or tuple(t.shape) != (h, w) or t.element_size() != isz or not t.is_contiguous():
                    raise ValueError(f"trace {i}: a contiguous host tensor of shape {(h, w)} expected")
                if stream is None:
                    stream = _current_stream(None)
                ptrs[i] = t.data_ptr()
            else:
                a = np.ascontiguousarray(t, dtype=dtype_of(self.field))
                if a.shape != (h, w):
                    raise ValueError(f"trace {i}: shape {a.shape}, expected {(h, w)}")
                keep.append(a)
                ptrs[i] = a.ctypes.data
        N.check(N.load().zkb_batch_run_host(self._h, ptrs, stream))

    def set_merkle_fusion(self, leaf_levels: int, comp_levels: int) -> None:
        """Persistent plans: Merkle levels the leaf tile computes above the leaves (0..8)
        and levels per compression tile (1..8)."""
        N.check(N.load().zkb_batch_set_merkle_fusion(self._h, leaf_levels, comp_levels))

    def queue_info(self) -> dict:
        q = N.BatchQueueInfo()
        N.check(N.load().zkb_batch_queue_info(self._h, C.byref(q)))
        return {k: int(getattr(q, k)) for k, _ in N.BatchQueueInfo._fields_}

    def profile(self, stream=None) -> dict:
        """One profiled run of a persistent plan: summed block-busy ms by item kind, span ms."""
        busy = (C.c_double * 4)()
        span = C.c_double()
        N.check(N.load().zkb_batch_profile(self._h, stream, busy, C.byref(span)))
        return {"pass_ms": busy[0], "fused_ms": busy[1], "leaf_ms": busy[2], "compress_ms": busy[3],
                "span_ms": span.value}

    def debug_stalled_run(self, spin_limit: int, stream=None) -> None:
        """One run whose work queue holds an item waiting on a counter nothing bumps: the
        kernel gives up after spin_limit polls and roots() then raises ZKB_ERR_TIMEOUT."""
        N.check(N.load().zkb_debug_batch_stalled_run(self._h, spin_limit, stream))

    def roots(self, stream=None) -> np.ndarray:
        out = np.zeros((len(self), self.digest_elems), dtype=dtype_of(self.field))
        N.check(N.load().zkb_batch_roots(self._h, _ptr(out), stream))
        return out

    def tree(self, i: int) -> Tree:
        t = C.c_void_p()
        N.check(N.load().zkb_batch_tree(self._h, i, C.byref(t)))
        h, w = self.shapes[i]
        return Tree(t, self.field, [(h << self.log_blowup, w)], owner=self)

    def info(self) -> dict:
        st = N.BatchInfo()
        N.check(N.load().zkb_batch_info(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in N.BatchInfo._fields_}

    def lde_tune(self, i: int) -> Tuple[int, int, int]:
        k, cp, cf = C.c_int(), C.c_uint32(), C.c_uint32()
        N.check(N.load().zkb_batch_lde_tune(self._h, i, C.byref(k), C.byref(cp), C.byref(cf)))
        return k.value, cp.value, cf.value

    def close(self):
        h = getattr(self, "_h", None)
        self._h = None
        if h:
            try:
                N.load().zkb_batch_free(h)
            except Exception:  # interpreter shutdown
                pass

    def __del__(self):
        self.close()


def _current_stream(t):
    """torch's current stream on the tensor's device (the current device for host tensors)."""
    import torch

    if t is None or not t.is_cuda:
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)
