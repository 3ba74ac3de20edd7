"""Full-size parity: the configurations' own sizes, every answer bit-exact.

The oracle's answers for these jobs are committed in tests/golden/fullsize.json, made
by tests/golden/make_fullsize.py from `bench.synthetic_trace` inputs (the same seeded
trace on every machine, the bench's own).  Each test regenerates the trace, runs the
job through the C ABI on the GPU and compares:

* BabyBear 2^22 x 256, blowup 2 — the bench's default job (zkb_pcs_commit_fri_dev):
  the trace root, every FRI beta and layer root, the 2^8 x 4 final codeword, the 100
  query indices, and SHA-256 digests of all query rows and sibling paths.
* Goldilocks 2^20 x 64, blowup 4 (2^22 rows, bit-reversed) — every LDE value (SHA-256
  of each block of 2^16 rows) and the MMCS roots with the width-16 / 8-element-digest
  and width-12 / 4-element-digest Poseidon2 hashers.

The semantics matched are p3's MerkleTree::new (vendor/p3-merkle-tree-gpu/src/
merkle_tree.rs:84-151), the coset LDE with bit-reversed rows
(zkf-backends/src/wrapping/stark_to_groth16.rs:2324-2346) and the fold
(stark_to_groth16.rs:2348-2371).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import bench
import ziros_b200 as Z

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fullsize.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _device_trace(torch, field, g):
    host = bench.synthetic_trace(field, 1 << g["log_rows"], g["width"], g["trace_seed"])
    view = host.view(np.int32 if field == 0 else np.int64)
    return torch.from_numpy(view).cuda()


def test_babybear_headline_job_matches_oracle(golden):
    import torch

    g = golden["babybear_2^22x256_b2"]
    fri = g["fri"]
    trace = _device_trace(torch, Z.BABYBEAR, g)
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, g["p2_seed"], g["log_blowup"])
    root, _, pf = pcs.commit_fri_dev(trace, g["alpha"], fri["log_final"], fri["num_queries"],
                                     fri["challenge_seed"], fri["query_seed"])
    del trace
    assert root.tolist() == g["root"]
    assert pf.rounds == g["log_rows"] + g["log_blowup"] - fri["log_final"] == len(g["fri_roots"])
    assert pf.betas.tolist() == g["fri_betas"]
    assert pf.roots.tolist() == g["fri_roots"]
    assert pf.final.tolist() == g["fri_final"]
    assert pf.query_indices.tolist() == g["query_indices"]
    assert pf.query_rows[0].tolist() == g["query0_rows"]
    assert _sha(pf.query_rows) == g["query_rows_sha256"]
    assert _sha(pf.query_siblings) == g["query_siblings_sha256"]


def test_goldilocks_config2_every_lde_value_and_roots(golden):
    import torch

    g = golden["goldilocks_2^20x64_b4"]
    n, w, lb = 1 << g["log_rows"], g["width"], g["log_blowup"]
    trace = _device_trace(torch, Z.GOLDILOCKS, g)
    out = torch.empty((n << lb, w), dtype=torch.int64, device="cuda")
    Z.CudaDft(Z.GOLDILOCKS).coset_lde_batch_dev(trace, lb, out, bit_reverse_rows=True)
    torch.cuda.synchronize()
    lde = out.cpu().numpy().view(np.uint64)
    del out
    br = g["block_rows"]
    got = [_sha(lde[r:r + br]) for r in range(0, lde.shape[0], br)]
    bad = [i for i, (a, b) in enumerate(zip(got, g["lde_block_sha256"])) if a != b]
    assert len(got) == len(g["lde_block_sha256"]) and not bad, f"LDE row blocks differ: {bad[:8]}"
    assert [str(int(x)) for x in lde[0]] == g["lde_row0"]
    del lde
    for p2w in (16, 12):
        root, _ = Z.CudaTwoAdicPcs(Z.GOLDILOCKS, g["p2_seed"], lb, p2w).commit_dev(trace, want_tree=False)
        assert [str(int(x)) for x in root] == g[f"root_w{p2w}"], f"width-{p2w} root differs"
