"""The CPU oracle against the reference's own vectors and against first principles.

These run without a GPU.  The oracle is the checker for every GPU parity test, so
it is pinned here before it is trusted: the reference's golden vectors
(tests/golden/reference_vectors.json) and independent Python-integer restatements
of the DFT, the coset LDE, the MMCS relations and the FRI fold.
"""
import json
import os

import numpy as np
import pytest

from conftest import BB_P, GL_P, rand_field

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))


def test_goldilocks_poseidon2_golden_vector(oracle):
    g = GOLD["poseidon2_goldilocks_w16_seed42"]
    rc, rf, rp = oracle.round_constants(oracle.GOLDILOCKS, g["seed"])
    assert (rf, rp) == (8, 22) and rc.size == 8 * 16 + 22
    out = oracle.permute(oracle.GOLDILOCKS, np.array(g["input"], dtype=np.uint64), rc, rf, rp)
    assert [int(x) for x in out] == [int(h, 16) for h in g["output_hex"]]
    # LE byte encoding (safety net 3 of the reference test)
    assert out.astype("<u8").tobytes() == b"".join(int(h, 16).to_bytes(8, "little") for h in g["output_hex"])


def test_dft_known_answer(oracle):
    g = GOLD["dft_basic_goldilocks"]
    out = oracle.dft_batch(oracle.GOLDILOCKS, np.array(g["input"], dtype=np.uint64).reshape(-1, 1))
    assert int(out[0, 0]) == g["output0"]


def test_external_mds_chunk(oracle):
    g = GOLD["external_mds_chunk"]
    st = np.zeros(16, dtype=np.uint64)
    st[:4] = g["input_prefix"]
    # zero rounds: the permutation reduces to the initial external linear layer
    out = oracle.permute(oracle.GOLDILOCKS, st, np.zeros(0, np.uint64), 0, 0)
    assert list(out[:4]) == g["output_prefix"]
    assert [int(out[i]) for i in range(4, 16)] == [g["others_mod4"][i % 4] for i in range(4, 16)]


def test_babybear_diagonal(oracle):
    d = oracle.diagonal(oracle.BABYBEAR)
    assert d[1] == 1 and d[2] == 2 and d[4] == 3 and d[5] == 4
    assert d[0] == BB_P - 2 and d[7] == BB_P - 3 and d[8] == BB_P - 4
    inv2 = pow(2, BB_P - 2, BB_P)
    assert d[3] == inv2 and d[12] == pow(inv2, 27, BB_P) and d[15] == BB_P - pow(inv2, 27, BB_P)
    assert all(int(x) < BB_P for x in d)


def test_constants_layout_and_determinism(oracle):
    for field, width, n in [(oracle.BABYBEAR, 16, 141), (oracle.GOLDILOCKS, 16, 150), (oracle.GOLDILOCKS, 12, 118)]:
        a, rf, rp = oracle.round_constants(field, 42, width)
        b, _, _ = oracle.round_constants(field, 42, width)
        c, _, _ = oracle.round_constants(field, 43, width)
        assert a.size == n == rf * width + rp
        assert (a == b).all() and not (a == c).all()
        p = BB_P if field == oracle.BABYBEAR else GL_P
        assert int(a.max()) < p


def test_two_adic_generators(oracle):
    assert oracle.two_adic_generator(oracle.GOLDILOCKS, 32) == 1753635133440165772
    assert oracle.two_adic_generator(oracle.BABYBEAR, 27) == 0x1A427A41
    for field, p, s in [(oracle.BABYBEAR, BB_P, 27), (oracle.GOLDILOCKS, GL_P, 32)]:
        for bits in (1, 5, s):
            g = oracle.two_adic_generator(field, bits)
            assert pow(g, 1 << bits, p) == 1 and pow(g, 1 << (bits - 1), p) == p - 1


def _naive_dft(col, p, w):
    n = len(col)
    return [sum(int(col[j]) * pow(w, j * k, p) for j in range(n)) % p for k in range(n)]


@pytest.mark.parametrize("field,p", [(0, BB_P), (1, GL_P)])
def test_dft_matches_definition(oracle, field, p):
    for log_n in (1, 3, 5):
        m = rand_field(field, (1 << log_n, 3), 11 + log_n)
        out = oracle.dft_batch(field, m)
        w = oracle.two_adic_generator(field, log_n)
        for c in range(3):
            assert [int(x) for x in out[:, c]] == _naive_dft(m[:, c], p, w)
        back = oracle.dft_batch(field, out, inverse=True)
        assert (back == m).all()


def _rev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


@pytest.mark.parametrize("field,p", [(0, BB_P), (1, GL_P)])
@pytest.mark.parametrize("log_n,log_b", [(3, 1), (3, 2), (2, 3), (0, 1)])
def test_coset_lde_matches_polynomial(oracle, field, p, log_n, log_b):
    n, N = 1 << log_n, 1 << (log_n + log_b)
    t = rand_field(field, (n, 2), 100 + log_n * 7 + log_b)
    lde = oracle.coset_lde(field, t, log_b)
    shift = oracle.field_generator(field)
    w_n = oracle.two_adic_generator(field, log_n)
    w_N = oracle.two_adic_generator(field, log_n + log_b)
    inv_n = pow(n, p - 2, p)
    for c in range(2):
        # interpolate over the subgroup: c_m = 1/n sum_j t_j w^-jm
        coef = [inv_n * sum(int(t[j, c]) * pow(w_n, (p - 2) * j * m, p) for j in range(n)) % p for m in range(n)]
        for i in range(N):
            x = shift * pow(w_N, _rev(i, log_n + log_b), p) % p
            assert int(lde[i, c]) == sum(cm * pow(x, m, p) for m, cm in enumerate(coef)) % p
    nat = oracle.coset_lde(field, t, log_b, bitrev=False)
    assert (nat[[_rev(i, log_n + log_b) for i in range(N)]] == lde).all()


def test_sponge_and_compress_relations(oracle):
    for field, width in [(oracle.BABYBEAR, 16), (oracle.GOLDILOCKS, 16), (oracle.GOLDILOCKS, 12)]:
        h = oracle.hasher(field, 42, width)
        rc, rf, rp = oracle.round_constants(field, 42, width)
        d = oracle.diagonal(field, width)
        dt = np.uint32 if field == 0 else np.uint64
        # empty input: no permutation, zero digest
        assert not oracle.sponge(h, np.zeros(0, dt)).any()
        # <= 8 elements: one permutation of the zero-padded state
        x = rand_field(field, 5, 3)
        st = np.zeros(width, dt)
        st[:5] = x
        assert (oracle.sponge(h, x) == oracle.permute(field, st, rc, rf, rp, width, d)[:h.out]).all()
        # 11 elements: second chunk overwrites lanes 0..2 only
        y = rand_field(field, 11, 4)
        st = np.zeros(width, dt)
        st[:8] = y[:8]
        st = oracle.permute(field, st, rc, rf, rp, width, d)
        st[:3] = y[8:]
        assert (oracle.sponge(h, y) == oracle.permute(field, st, rc, rf, rp, width, d)[:h.out]).all()
        # compress = truncated permutation of left || right
        l, r = rand_field(field, h.out, 5), rand_field(field, h.out, 6)
        st = np.zeros(width, dt)
        st[:h.out], st[h.out:2 * h.out] = l, r
        assert (oracle.compress(h, l, r) == oracle.permute(field, st, rc, rf, rp, width, d)[:h.out]).all()


def test_mmcs_structure(oracle):
    h = oracle.hasher(oracle.BABYBEAR, 42)
    m = rand_field(0, (4, 9), 1)
    layers = oracle.mmcs_commit(h, [m])
    leaves = [oracle.sponge(h, m[i]) for i in range(4)]
    assert all((layers[0][i] == leaves[i]).all() for i in range(4))
    root = oracle.compress(h, oracle.compress(h, leaves[0], leaves[1]), oracle.compress(h, leaves[2], leaves[3]))
    assert (layers[-1][0] == root).all()
    # odd height: padded with a zero digest, never hashed
    m3 = rand_field(0, (3, 4), 2)
    l3 = oracle.mmcs_commit(h, [m3])
    assert len(l3[0]) == 4 and not l3[0][3].any()
    # mixed heights: the 2-row matrix is injected one layer up
    big, small = rand_field(0, (4, 3), 3), rand_field(0, (2, 5), 4)
    lm = oracle.mmcs_commit(h, [small, big])
    lb = [oracle.sponge(h, big[i]) for i in range(4)]
    n0 = oracle.compress(h, oracle.compress(h, lb[0], lb[1]), oracle.sponge(h, small[0]))
    n1 = oracle.compress(h, oracle.compress(h, lb[2], lb[3]), oracle.sponge(h, small[1]))
    assert (lm[-1][0] == oracle.compress(h, n0, n1)).all()
    # two tallest matrices share one leaf hash over the concatenated rows (commit order)
    a, b = rand_field(0, (4, 3), 5), rand_field(0, (4, 6), 6)
    lab = oracle.mmcs_commit(h, [a, b])
    assert (lab[0][2] == oracle.sponge(h, np.concatenate([a[2], b[2]]))).all()


def test_mmcs_open_verify(oracle):
    h = oracle.hasher(oracle.GOLDILOCKS, 7)
    m = rand_field(1, (16, 10), 9)
    layers = oracle.mmcs_commit(h, [m])
    for idx in (0, 5, 15):
        rows, proof = oracle.mmcs_open(layers, [m], idx)
        node, i = oracle.sponge(h, rows[0]), idx
        for sib in proof:
            node = oracle.compress(h, node, sib) if i % 2 == 0 else oracle.compress(h, sib, node)
            i >>= 1
        assert (node == layers[-1][0]).all()


def _ext_mul(a, b):
    c = [0] * 7
    for i in range(4):
        for j in range(4):
            c[i + j] += int(a[i]) * int(b[j])
    return [(c[k] + 11 * (c[k + 4] if k + 4 < 7 else 0)) % BB_P for k in range(4)]


def test_ext4_arithmetic(oracle):
    a, b, c = rand_field(0, 4, 1), rand_field(0, 4, 2), rand_field(0, 4, 3)
    assert list(oracle.bb4_mul(a, b)) == _ext_mul(a, b)
    assert (oracle.bb4_mul(oracle.bb4_mul(a, b), c) == oracle.bb4_mul(a, oracle.bb4_mul(b, c))).all()
    x = np.array([0, 1, 0, 0], np.uint32)
    x4 = oracle.bb4_mul(oracle.bb4_mul(x, x), oracle.bb4_mul(x, x))
    assert list(x4) == [11, 0, 0, 0]


def test_fri_fold_p3_forms(oracle):
    """fold_matrix (coefficient form) equals fold_row (interpolation through (s, e0), (-s, e1))."""
    n_out = 16
    ev = rand_field(0, (2 * n_out, 4), 12)
    beta = rand_field(0, 4, 13)
    out = oracle.fri_fold_ext4(ev, beta)
    log_n = 4
    g = oracle.two_adic_generator(0, log_n + 1)
    for i in range(n_out):
        s = pow(g, _rev(i, log_n), BB_P)
        e0, e1 = [int(x) for x in ev[2 * i]], [int(x) for x in ev[2 * i + 1]]
        # e0 + (beta - s) * (e1 - e0) / (-s - s)
        inv = pow((BB_P - 2 * s) % BB_P, BB_P - 2, BB_P)
        bm = [(int(beta[0]) - s) % BB_P] + [int(x) for x in beta[1:]]
        diff = [(e1[k] - e0[k]) % BB_P for k in range(4)]
        t = _ext_mul(bm, diff)
        assert [int(x) for x in out[i]] == [(e0[k] + t[k] * inv) % BB_P for k in range(4)]
    # a base-field beta reduces the extension fold to the base fold with p3 twiddles
    evb = rand_field(0, 2 * n_out, 14)
    alpha = 123456
    base = oracle.fri_fold_base(0, evb, alpha, oracle.fri_inv_twiddles(0, n_out))
    ext_in = np.zeros((2 * n_out, 4), np.uint32)
    ext_in[:, 0] = evb
    ext = oracle.fri_fold_ext4(ext_in, np.array([alpha, 0, 0, 0], np.uint32))
    assert (ext[:, 0] == base).all() and not ext[:, 1:].any()


def test_fri_reference_fixture(oracle):
    g = GOLD["fri_fold_goldilocks_fixture"]
    n = g["n_output"]
    ev = np.array([(i * 7 + 1) % GL_P for i in range(2 * n)], np.uint64)
    tw = np.array([(i * 13 + 3) % GL_P for i in range(n)], np.uint64)
    out = oracle.fri_fold_base(1, ev, g["alpha"], tw)
    inv2 = (GL_P + 1) // 2
    for i in (0, 1, 777, n - 1):
        e, o = int(ev[2 * i]), int(ev[2 * i + 1])
        want = ((e + o) * inv2 + (e - o) * int(tw[i]) * g["alpha"]) % GL_P
        assert int(out[i]) == want


def test_fri_commit_oracle_relations(oracle):
    """The oracle's FRI commit phase: round-0 leaves are the codeword pairs, each opened
    path hashes to its round's root, and folding a degree-<2^k codeword (a polynomial
    evaluated on the bit-reversed subgroup) halves the degree bound."""
    cw = rand_field(0, (64, 4), 1)
    res = oracle.fri_commit_ext4(cw, 2, 42, 7, 4, 9)
    h = oracle.hasher(0, 42)
    assert res["roots"].shape == (4, 8) and res["final"].shape == (4, 4)
    for q, per_round in zip(res["indices"], res["queries"]):
        for r, (row, proof) in enumerate(per_round):
            node, i = oracle.sponge(h, row), (int(q) >> r) >> 1
            for sib in proof:
                node = oracle.compress(h, node, sib) if i % 2 == 0 else oracle.compress(h, sib, node)
                i >>= 1
            assert (node == res["roots"][r]).all()

