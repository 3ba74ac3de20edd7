"""ctypes wrapper of the CPU oracle (liboracle.so, built from oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, by ``__graft_entry__.smoke()`` and by
the CPU-baseline legs of ``bench.py`` as the parity checker.  The product
package (``ziros_b200``) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

BABYBEAR = 0
GOLDILOCKS = 1
BB_P = 0x78000001
GL_P = 0xFFFFFFFF00000001

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


class Hasher(C.Structure):
    _fields_ = [
        ("field", C.c_int),
        ("width", C.c_int),
        ("rate", C.c_int),
        ("out", C.c_int),
        ("rounds_f", C.c_int),
        ("rounds_p", C.c_int),
        ("rc", C.c_uint64 * 512),
        ("diag", C.c_uint64 * 16),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        sz = C.c_size_t
        u64 = C.c_uint64
        sig = {
            "or_bb_mul": (C.c_uint32, [C.c_uint32, C.c_uint32]),
            "or_gl_mul": (u64, [u64, u64]),
            "or_two_adic_generator": (u64, [C.c_int, C.c_int]),
            "or_field_generator": (u64, [C.c_int]),
            "or_rng_fill_u64": (None, [u64, P, sz]),
            "or_rng_fill_bb": (None, [u64, P, sz]),
            "or_combine_columns_ext4": (None, [P, sz, sz, P, P]),
            "or_p2_round_numbers": (C.c_int, [C.c_int, C.c_int, P, P]),
            "or_p2_constants_bb": (C.c_int, [u64, C.c_int, P, sz]),
            "or_p2_constants_gl": (C.c_int, [u64, C.c_int, P, sz]),
            "or_p2_diag_bb16": (None, [P]),
            "or_p2_diag_gl16": (None, [P]),
            "or_p2_diag_gl12": (None, [P]),
            "or_p2_permute_bb": (None, [P, sz, C.c_int, P, C.c_int, C.c_int, P]),
            "or_p2_permute_gl": (None, [P, sz, C.c_int, P, C.c_int, C.c_int, P]),
            "or_hasher_init": (C.c_int, [P, C.c_int, C.c_int, u64]),
            "or_sponge": (None, [P, P, sz, P]),
            "or_compress": (None, [P, P, P, P]),
            "or_hash_rows": (None, [P, P, P, sz, sz, P]),
            "or_mmcs_commit": (C.c_int, [P, P, P, P, sz, P, sz, P, C.c_int]),
            "or_mmcs_layers_total": (sz, [sz]),
            "or_dft_batch": (None, [C.c_int, P, C.c_int, sz, C.c_int]),
            "or_coset_lde_batch": (None, [C.c_int, P, C.c_int, sz, C.c_int, u64, C.c_int, P]),
            "or_bit_reverse_rows": (None, [C.c_int, P, C.c_int, sz]),
            "or_fri_fold_base": (None, [C.c_int, P, sz, u64, P, P]),
            "or_fri_fold_ext4": (None, [P, sz, P, P]),
            "or_fri_inv_twiddles": (None, [C.c_int, sz, P]),
            "or_bb4_mul": (None, [P, P, P]),
            "or_num_threads": (C.c_int, []),
            "or_set_threads": (None, [C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def dtype_of(field: int):
    return np.uint32 if field == BABYBEAR else np.uint64


# ---------------------------------------------------------------- fields / rng
def two_adic_generator(field: int, bits: int) -> int:
    return int(lib().or_two_adic_generator(field, bits))


def field_generator(field: int) -> int:
    return int(lib().or_field_generator(field))


def rng_u64(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    lib().or_rng_fill_u64(seed, _ptr(out), n)
    return out


# ------------------------------------------------------------------- poseidon2
def round_numbers(field: int, width: int = 16):
    rf, rp = C.c_int(), C.c_int()
    if lib().or_p2_round_numbers(field, width, C.byref(rf), C.byref(rp)):
        raise ValueError("unsupported Poseidon2 width")
    return rf.value, rp.value


def round_constants(field: int, seed: int, width: int = 16):
    """flatten_round_constants(seed) -> (flat, rounds_f, rounds_p)."""
    rf, rp = round_numbers(field, width)
    n = rf * width + rp
    out = np.zeros(n, dtype=dtype_of(field))
    fn = lib().or_p2_constants_bb if field == BABYBEAR else lib().or_p2_constants_gl
    if fn(seed, width, _ptr(out), n) != n:
        raise RuntimeError("constant generation failed")
    return out, rf, rp


def diagonal(field: int, width: int = 16) -> np.ndarray:
    out = np.zeros(width, dtype=dtype_of(field))
    if field == BABYBEAR and width == 16:
        lib().or_p2_diag_bb16(_ptr(out))
    elif field == GOLDILOCKS and width == 16:
        lib().or_p2_diag_gl16(_ptr(out))
    elif field == GOLDILOCKS and width == 12:
        lib().or_p2_diag_gl12(_ptr(out))
    else:
        raise ValueError("no diagonal for this field/width")
    return out


def permute(field: int, states: np.ndarray, rc: np.ndarray, rf: int, rp: int,
            width: int = 16, diag: np.ndarray | None = None) -> np.ndarray:
    s = np.ascontiguousarray(states, dtype=dtype_of(field)).copy()
    d = diagonal(field, width) if diag is None else np.ascontiguousarray(diag, dtype=dtype_of(field))
    rc = np.ascontiguousarray(rc, dtype=dtype_of(field))
    fn = lib().or_p2_permute_bb if field == BABYBEAR else lib().or_p2_permute_gl
    fn(_ptr(s), s.size // width, width, _ptr(rc), rf, rp, _ptr(d))
    return s


def hasher(field: int, seed: int, width: int = 16) -> Hasher:
    h = Hasher()
    if lib().or_hasher_init(C.byref(h), field, width, seed):
        raise ValueError("unsupported hasher configuration")
    return h


def sponge(h: Hasher, elems: np.ndarray) -> np.ndarray:
    e = np.ascontiguousarray(elems, dtype=dtype_of(h.field))
    out = np.zeros(h.out, dtype=dtype_of(h.field))
    lib().or_sponge(C.byref(h), _ptr(e), e.size, _ptr(out))
    return out


def compress(h: Hasher, left: np.ndarray, right: np.ndarray) -> np.ndarray:
    dt = dtype_of(h.field)
    l = np.ascontiguousarray(left, dtype=dt)
    r = np.ascontiguousarray(right, dtype=dt)
    out = np.zeros(h.out, dtype=dt)
    lib().or_compress(C.byref(h), _ptr(l), _ptr(r), _ptr(out))
    return out


def hash_rows(h: Hasher, mats) -> np.ndarray:
    mats = [np.ascontiguousarray(m, dtype=dtype_of(h.field)) for m in mats]
    height = mats[0].shape[0]
    ptrs = (C.c_void_p * len(mats))(*[m.ctypes.data for m in mats])
    widths = (C.c_size_t * len(mats))(*[m.shape[1] for m in mats])
    out = np.zeros((height, h.out), dtype=dtype_of(h.field))
    lib().or_hash_rows(C.byref(h), ptrs, widths, len(mats), height, _ptr(out))
    return out


def mmcs_commit(h: Hasher, mats):
    """p3 MerkleTree::new over row-major matrices -> list of digest layers (root last)."""
    mats = [np.ascontiguousarray(m, dtype=dtype_of(h.field)) for m in mats]
    n = len(mats)
    ptrs = (C.c_void_p * n)(*[m.ctypes.data for m in mats])
    heights = (C.c_size_t * n)(*[m.shape[0] for m in mats])
    widths = (C.c_size_t * n)(*[m.shape[1] for m in mats])
    max_h = max(m.shape[0] for m in mats)
    total = lib().or_mmcs_layers_total(max_h) * h.out
    buf = np.zeros(total, dtype=dtype_of(h.field))
    lens = (C.c_size_t * 80)()
    nl = lib().or_mmcs_commit(C.byref(h), ptrs, heights, widths, n, _ptr(buf), total, lens, 80)
    if nl < 0:
        raise ValueError("mmcs commit rejected the matrices")
    layers, off = [], 0
    for i in range(nl):
        k = lens[i] * h.out
        layers.append(buf[off:off + k].reshape(lens[i], h.out).copy())
        off += k
    return layers


def mmcs_open(layers, mats, index: int):
    """Mmcs::open_batch: rows of every matrix at the reduced index, sibling path."""
    max_h = max(m.shape[0] for m in mats)
    log_max = (max_h - 1).bit_length()
    rows = []
    for m in mats:
        lh = (m.shape[0] - 1).bit_length()
        rows.append(np.array(m[index >> (log_max - lh)]))
    proof = [layers[i][(index >> i) ^ 1] for i in range(log_max)]
    return rows, proof


# ------------------------------------------------------------------------ DFT
def dft_batch(field: int, mat: np.ndarray, inverse: bool = False) -> np.ndarray:
    m = np.ascontiguousarray(mat, dtype=dtype_of(field)).copy()
    h = m.shape[0]
    w = m.shape[1] if m.ndim == 2 else 1
    lib().or_dft_batch(field, _ptr(m), h.bit_length() - 1, w, int(inverse))
    return m


def coset_lde(field: int, trace: np.ndarray, log_blowup: int, shift: int | None = None,
              bitrev: bool = True) -> np.ndarray:
    t = np.ascontiguousarray(trace, dtype=dtype_of(field))
    h, w = t.shape
    if shift is None:
        shift = field_generator(field)
    out = np.zeros((h << log_blowup, w), dtype=dtype_of(field))
    lib().or_coset_lde_batch(field, _ptr(t), h.bit_length() - 1, w, log_blowup, shift,
                             int(bitrev), _ptr(out))
    return out


# ------------------------------------------------------------------------ FRI
def fri_fold_base(field: int, evals: np.ndarray, alpha: int, inv_tw: np.ndarray) -> np.ndarray:
    e = np.ascontiguousarray(evals, dtype=dtype_of(field))
    t = np.ascontiguousarray(inv_tw, dtype=dtype_of(field))
    out = np.zeros(e.size // 2, dtype=dtype_of(field))
    lib().or_fri_fold_base(field, _ptr(e), out.size, alpha, _ptr(t), _ptr(out))
    return out


def fri_inv_twiddles(field: int, n_out: int) -> np.ndarray:
    out = np.zeros(n_out, dtype=dtype_of(field))
    lib().or_fri_inv_twiddles(field, n_out, _ptr(out))
    return out


def fri_fold_ext4(evals: np.ndarray, beta) -> np.ndarray:
    e = np.ascontiguousarray(evals, dtype=np.uint32).reshape(-1, 4)
    b = np.ascontiguousarray(beta, dtype=np.uint32)
    out = np.zeros((e.shape[0] // 2, 4), dtype=np.uint32)
    lib().or_fri_fold_ext4(_ptr(e), out.shape[0], _ptr(b), _ptr(out))
    return out


def bb4_mul(a, b) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().or_bb4_mul(_ptr(a), _ptr(b), _ptr(out))
    return out


def num_threads() -> int:
    return int(lib().or_num_threads())


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def rng_bb(seed: int, n: int) -> np.ndarray:
    """n BabyBear draws (p3 sampler) from SmallRng(seed)."""
    out = np.empty(n, dtype=np.uint32)
    lib().or_rng_fill_bb(seed, _ptr(out), n)
    return out


def combine_columns_ext4(lde: np.ndarray, alpha) -> np.ndarray:
    m = np.ascontiguousarray(lde, dtype=np.uint32)
    a = np.ascontiguousarray(alpha, dtype=np.uint32)
    out = np.zeros((m.shape[0], 4), dtype=np.uint32)
    lib().or_combine_columns_ext4(_ptr(m), m.shape[0], m.shape[1], _ptr(a), _ptr(out))
    return out


class DuplexChallenger:
    """p3 DuplexChallenger<F, Poseidon2<16>, 16, 8>, restated from
    zkf-backends/src/wrapping/duplex_challenger.rs:1-145 (which mirrors p3-challenger):
    observe() clears the output buffer and duplexes when 8 inputs are pending; sample()
    duplexes when input is pending or no output is left and pops the LAST output;
    duplexing overwrites state[0..len(input)], permutes, outputs state[0..8].
    sample_bits(b) masks a sample to b bits (stark_to_groth16.rs:2229-2255)."""

    def __init__(self, field: int, p2_seed: int):
        self.field = field
        self.rc, self.rf, self.rp = round_constants(field, p2_seed, 16)
        self.state = np.zeros(16, dtype=dtype_of(field))
        self.inp, self.out = [], []

    def _duplex(self):
        for i, v in enumerate(self.inp):
            self.state[i] = v
        self.inp = []
        self.state = permute(self.field, self.state, self.rc, self.rf, self.rp, 16)
        self.out = [int(x) for x in self.state[:8]]

    def observe(self, values):
        for v in np.atleast_1d(values):
            self.out = []
            self.inp.append(int(v))
            if len(self.inp) == 8:
                self._duplex()

    def sample(self, n: int = 1) -> np.ndarray:
        res = []
        for _ in range(n):
            if self.inp or not self.out:
                self._duplex()
            res.append(self.out.pop())
        return np.array(res, dtype=np.uint64)

    def sample_bits(self, bits: int) -> int:
        return int(self.sample(1)[0]) & ((1 << bits) - 1)


def fri_commit_ext4(codeword: np.ndarray, log_final: int, p2_seed: int, challenge_seed: int,
                    num_queries: int, query_seed: int, challenger: DuplexChallenger | None = None) -> dict:
    """FRI commit phase (p3 commit_phase/answer_query restated): round r commits the
    codeword as rows of (x, -x) pairs flattened to 8 base elements, then folds with
    beta_r; queries open row (index >> r) >> 1 of every round.  Challenges: seeded
    draws, or with `challenger` the transcript (observe root r, sample beta_r; observe
    the final codeword; query index = sample_bits(log_n))."""
    cw = np.ascontiguousarray(codeword, dtype=np.uint32).reshape(-1, 4)
    log_n = cw.shape[0].bit_length() - 1
    rounds = log_n - log_final
    h = hasher(BABYBEAR, p2_seed)
    betas = rng_bb(challenge_seed, 4 * rounds).reshape(rounds, 4) if challenger is None else \
        np.zeros((rounds, 4), np.uint32)
    trees, leaves = [], []
    cur = cw
    for r in range(rounds):
        mat = cur.reshape(-1, 8)
        layers = mmcs_commit(h, [mat])
        trees.append(layers)
        leaves.append(mat)
        if challenger is not None:
            challenger.observe(layers[-1][0])
            betas[r] = challenger.sample(4).astype(np.uint32)
        cur = fri_fold_ext4(cur, betas[r])
    if challenger is None:
        idx = (rng_u64(query_seed, num_queries) >> np.uint64(64 - log_n)).astype(np.uint64)
    else:
        challenger.observe(cur.reshape(-1))
        idx = np.array([challenger.sample_bits(log_n) for _ in range(num_queries)], dtype=np.uint64)
    queries = []
    for q in idx:
        per_round = []
        for r in range(rounds):
            pair = (int(q) >> r) >> 1
            rows, proof = mmcs_open(trees[r], [leaves[r]], pair)
            per_round.append((rows[0], proof))
        queries.append(per_round)
    return {"roots": np.array([t[-1][0] for t in trees]), "betas": betas, "final": cur,
            "indices": idx, "queries": queries}


# ------------------------------------------------------------------ polynomial ops
def poly_eval_gl(coeffs, points) -> np.ndarray:
    """Horner evaluation (zkf-metal/src/poly.rs:276-283 horner_eval), Python integers."""
    p = GL_P
    out = []
    for x in points:
        r = 0
        for c in reversed([int(v) for v in coeffs]):
            r = (r * int(x) + c) % p
        out.append(r)
    return np.array(out, dtype=np.uint64)


def poly_coset_eval_gl(coeffs, shift: int, log_n: int) -> np.ndarray:
    """f(shift * w^i) for i < 2^log_n, w = two_adic_generator(log_n) (poly.rs:337-363)."""
    p = GL_P
    w = int(two_adic_generator(1, log_n))
    pts = [(shift * pow(w, i, p)) % p for i in range(1 << log_n)]
    return poly_eval_gl(coeffs, pts)


def poly_quotient_gl(evals, z: int, f_z: int) -> np.ndarray:
    """(e_i - f_z) / (w^i - z) on the subgroup, 0 where w^i = z (poly.rs:366-400)."""
    p = GL_P
    n = len(evals)
    w = int(two_adic_generator(1, n.bit_length() - 1))
    out = []
    x = 1
    for e in evals:
        d = (x - z) % p
        out.append(0 if d == 0 else ((int(e) - f_z) % p) * pow(d, p - 2, p) % p)
        x = x * w % p
    return np.array(out, dtype=np.uint64)
