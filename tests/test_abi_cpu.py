"""C-ABI checks that need no GPU: the library loads, exports every symbol that
include/zkb200.h declares, and its host-side logic (Poseidon2 constant
generation, argument validation, the no-device decline) behaves."""
import os
import re

import numpy as np
import pytest

import ziros_b200 as Z
from ziros_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "zkb200.h")).read()
    return sorted(set(re.findall(r"ZKB_API[^;(]*?\b(zkb_\w+)\s*\(", text)))


def test_header_declares_exported_symbols():
    syms = header_symbols()
    assert len(syms) >= 20
    lib = N.load()
    for s in syms:
        assert hasattr(lib, s), s
    # the ctypes table covers exactly the header
    assert sorted(N.SIGNATURES) == syms


def test_exported_symbols_in_dynamic_table():
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (zkb_\w+)", out))
    assert set(header_symbols()) <= exported


@pytest.mark.parametrize("field,width", [(Z.BABYBEAR, 16), (Z.GOLDILOCKS, 16), (Z.GOLDILOCKS, 12)])
@pytest.mark.parametrize("seed", [0, 42, 0xDEADBEEFCAFEF00D])
def test_round_constants_match_oracle(oracle, field, width, seed):
    ours, ne, ni = Z.round_constants(field, seed, width)
    ref, rf, rp = oracle.round_constants(field, seed, width)
    assert (ne, ni) == (rf, rp)
    assert (ours == ref).all()


def test_round_constants_capacity_error():
    lib = N.load()
    import ctypes as C

    buf = np.zeros(4, np.uint32)
    rc = lib.zkb_poseidon2_babybear_round_constants(1, buf.ctypes.data_as(C.c_void_p), 4, None, None)
    assert rc == N.ERR_INVALID
    assert "capacity" in N.last_error()


def test_version_and_errors_are_strings():
    assert N.load().zkb_version().startswith(b"zkb200")
    assert isinstance(N.last_error(), str)


@pytest.mark.skipif(N.device_count() > 0, reason="exercises the no-device decline path")
def test_no_device_declines():
    assert Z.CudaPoseidon2.new() is None
    assert Z.CudaFri.new() is None
    p = Z.CudaPoseidon2()
    rc, ne, ni = Z.round_constants(Z.BABYBEAR, 1)
    assert p.batch_permute_babybear(np.zeros(16, np.uint32), rc, ne, ni) is False
    assert "no CUDA device" in N.last_error()
    with pytest.raises(N.ZkbDeclined):
        Z.CudaDft(Z.GOLDILOCKS).dft_batch(np.arange(8, dtype=np.uint64))


@pytest.mark.parametrize("field", [0, 1])
def test_challenger_matches_oracle(oracle, field):
    """The transcript (DuplexChallenger) runs on the host and needs no device: observe /
    sample / sample_bits sequences equal the oracle's restatement, including observes
    that fill the rate exactly, interleaved samples and more samples than the rate."""
    import numpy as np

    import ziros_b200 as Z

    a, b = oracle.DuplexChallenger(field, 42), Z.Challenger(field, 42)
    script = [(1, 2, 3, 4, 5), (), tuple(range(8)), (9,) * 9, (100, 200, 300), (), (400, 500), tuple(range(20))]
    for obs in script:
        if obs:
            a.observe(np.array(obs))
            b.observe(np.array(obs))
        assert (a.sample(3) == b.sample(3)).all()
        assert (a.sample(9) == b.sample(9)).all()
        assert a.sample_bits(22) == b.sample_bits(22)


def test_challenger_rejects_non_canonical():
    import ziros_b200 as Z

    c = Z.Challenger(0, 1)
    with pytest.raises(Z.ZkbError):
        c.observe([0x78000001])


@pytest.mark.parametrize("field,p2w,shapes", [
    (0, 16, [(64, 16)]),
    (0, 16, [(37, 9), (19, 3), (5, 20), (37, 2)]),      # odd heights, injection, equal heights
    (1, 16, [(128, 8), (32, 5)]),
    (1, 12, [(16, 7), (8, 1), (2, 3)]),
])
def test_verify_batch_accepts_openings_and_rejects_tampering(oracle, field, p2w, shapes):
    """Mmcs::verify_batch (host-side, no device) against openings of the oracle's trees."""
    import numpy as np

    import ziros_b200 as Z
    from conftest import BB_P, GL_P, rand_field

    mats = [rand_field(field, s, 40 + i) for i, s in enumerate(shapes)]
    layers = oracle.mmcs_commit(oracle.hasher(field, 42, p2w), mats)
    root = layers[-1][0]
    mmcs = Z.CudaMerkleTreeMmcs(field, 42, p2w)
    max_h = max(h for h, _ in shapes)
    for index in sorted({0, max_h - 1, max_h // 2, 3 % max_h}):
        rows, proof = oracle.mmcs_open(layers, mats, index)
        assert mmcs.verify_batch(root, shapes, index, rows, proof)
        bad_rows = [r.copy() for r in rows]
        bad_rows[-1][0] = (int(bad_rows[-1][0]) + 1) % (BB_P if field == 0 else GL_P)
        assert not mmcs.verify_batch(root, shapes, index, bad_rows, proof)
        if proof:
            bad_proof = [p.copy() for p in proof]
            bad_proof[-1][0] ^= 1
            assert not mmcs.verify_batch(root, shapes, index, rows, bad_proof)
            assert not mmcs.verify_batch(root, shapes, index ^ 1, rows, proof) or index ^ 1 >= max_h
    if max_h > 1:  # a proof with the wrong number of siblings is rejected
        assert not mmcs.verify_batch(root, shapes, 0, oracle.mmcs_open(layers, mats, 0)[0], [])


def test_kill_switch_declines_every_call():
    """ZKB_DISABLE=1 (the reference's ZKF_METAL kill switch): entry points decline with
    that reason, before any device is looked for."""
    import subprocess
    import sys

    code = ("import numpy as np, ziros_b200 as Z\n"
            "from ziros_b200 import _native as N\n"
            "t = np.zeros((16, 4), np.uint32)\n"
            "try:\n"
            "    Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1).commit(t)\n"
            "    print('ran')\n"
            "except N.ZkbDeclined as e:\n"
            "    print('declined', e)\n")
    env = dict(os.environ, ZKB_DISABLE="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120,
                         cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert out.returncode == 0, out.stderr
    assert out.stdout.startswith("declined") and "ZKB_DISABLE" in out.stdout


def test_fault_injection_rejects_unknown_kinds():
    with pytest.raises(Z.ZkbError):
        N.inject_fault(7, 1)
    N.inject_fault(1, 0)
    assert N.circuit_open() == (False, "")


def test_thresholds_roundtrip_and_environment():
    N.set_thresholds(ntt=4096, poseidon2=1000, merkle=2048, fri=1024)
    assert N.get_thresholds() == {"ntt": 4096, "poseidon2": 1000, "merkle": 2048, "fri": 1024}
    N.set_thresholds()
    assert N.get_thresholds() == {"ntt": 0, "poseidon2": 0, "merkle": 0, "fri": 0}
    import subprocess
    import sys

    code = "from ziros_b200 import _native as N; print(N.get_thresholds())"
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ, ZKB_THRESHOLDS="ntt=512,merkle=64"),
                         cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == str({"ntt": 512, "poseidon2": 0, "merkle": 64, "fri": 0})


@pytest.mark.parametrize("field,p2w", [(0, 16), (1, 16), (1, 12)])
def test_compress_matches_oracle(oracle, field, p2w):
    """zkb_mmcs_compress (host-side, no device): TruncatedPermutation of digest pairs."""
    import numpy as np

    import ziros_b200 as Z
    from conftest import rand_field

    mmcs = Z.CudaMerkleTreeMmcs(field, 42, p2w)
    d = mmcs.digest_elems
    left, right = rand_field(field, (5, d), 1), rand_field(field, (5, d), 2)
    got = mmcs.compress(left, right)
    h = oracle.hasher(field, 42, p2w)
    assert np.array_equal(got, np.stack([oracle.compress(h, a, b) for a, b in zip(left, right)]))
    with pytest.raises(Z.ZkbError):
        bad = left.copy()
        bad[0, 0] = 0x78000001 if field == 0 else 0xFFFFFFFF00000001
        mmcs.compress(bad, right)
