#!/usr/bin/env python
"""Writes tests/golden/fullsize.json: the oracle's answers for the full-size jobs.

The inputs are `bench.synthetic_trace` draws (host-deterministic, the bench's own
trace), so the GPU tests and bench.py regenerate the same trace on any machine and
compare the device's answers with these fixtures word for word:

* babybear_2^22x256_b2 — the bench's default job: coset LDE x2 with bit-reversed rows,
  Poseidon2-W16 MMCS (seed 42), alpha-reduction of the LDE columns into one F_p^4
  codeword, FRI commit phase 2^23 -> 2^8 with 100 seeded queries.  Stored: the trace
  root, every FRI beta and root, the final codeword, the query indices, and SHA-256
  digests of the query rows and sibling paths (in the FriProof array layout).
* goldilocks_2^20x64_b4 — coset LDE x4 (2^22 rows, bit-reversed): SHA-256 of every
  block of 2^16 LDE rows (so every LDE value is compared), and the MMCS roots with the
  width-16 (8-element digest) and width-12 (4-element digest) Poseidon2 hashers.

Run on the host cores (oracle/ C restatement, OpenMP); about 10 minutes on 8 cores:
    python tests/golden/make_fullsize.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "fullsize.json")
BLOCK_ROWS = 1 << 16


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def block_digests(lde: np.ndarray, block_rows: int = BLOCK_ROWS) -> list:
    return [sha(lde[r:r + block_rows]) for r in range(0, lde.shape[0], block_rows)]


def fri_arrays(want: dict, log_n: int, nq: int):
    """The oracle's query answers in the FriProof layout: rows (nq, rounds, 8) and
    siblings (nq, sum over rounds of (log_n - r - 1) * 8)."""
    rounds = len(want["roots"])
    rows = np.zeros((nq, rounds, 8), np.uint32)
    sib = np.zeros((nq, sum(log_n - r - 1 for r in range(rounds)) * 8), np.uint32)
    for q in range(nq):
        off = 0
        for r in range(rounds):
            row, proof = want["queries"][q][r]
            rows[q, r] = row
            p = np.array(proof, np.uint32).reshape(-1)
            sib[q, off:off + p.size] = p
            off += p.size
    return rows, sib


def babybear_headline() -> dict:
    wl = bench.WORKLOADS["babybear_2^22x256_b2"]
    lh, w, lb = wl["log_h"], wl["width"], wl["log_blowup"]
    fri = bench.FRI
    trace = bench.synthetic_trace(0, 1 << lh, w, bench.TRACE_SEED)
    t0 = time.time()
    lde = O.coset_lde(O.BABYBEAR, trace, lb)
    del trace
    layers = O.mmcs_commit(O.hasher(O.BABYBEAR, bench.P2_SEED), [lde])
    root = layers[-1][0]
    del layers
    cw = O.combine_columns_ext4(lde, np.array(bench.ALPHA, np.uint32))
    del lde
    want = O.fri_commit_ext4(cw, fri["log_final"], bench.P2_SEED, fri["challenge_seed"], fri["num_queries"],
                             fri["query_seed"])
    rows, sib = fri_arrays(want, lh + lb, fri["num_queries"])
    print(f"babybear headline: {time.time() - t0:.0f} s", flush=True)
    return {
        "workload": "babybear_2^22x256_b2", "trace_seed": bench.TRACE_SEED, "log_rows": lh, "width": w,
        "log_blowup": lb, "p2_seed": bench.P2_SEED, "alpha": list(bench.ALPHA), "fri": dict(fri),
        "root": [int(x) for x in root],
        "fri_betas": want["betas"].astype(np.uint32).tolist(),
        "fri_roots": want["roots"].astype(np.uint32).tolist(),
        "fri_final": want["final"].astype(np.uint32).tolist(),
        "query_indices": [int(x) for x in want["indices"]],
        "query_rows_sha256": sha(rows), "query_siblings_sha256": sha(sib),
        "query0_rows": rows[0].tolist(),
    }


def goldilocks_lde() -> dict:
    wl = bench.WORKLOADS["goldilocks_2^20x64_b4"]
    lh, w, lb = wl["log_h"], wl["width"], wl["log_blowup"]
    trace = bench.synthetic_trace(1, 1 << lh, w, bench.TRACE_SEED)
    t0 = time.time()
    lde = O.coset_lde(O.GOLDILOCKS, trace, lb)
    out = {"workload": "goldilocks_2^20x64_b4", "trace_seed": bench.TRACE_SEED, "log_rows": lh, "width": w,
           "log_blowup": lb, "p2_seed": bench.P2_SEED, "block_rows": BLOCK_ROWS,
           "lde_block_sha256": block_digests(lde), "lde_row0": [str(int(x)) for x in lde[0]]}
    for p2w in (16, 12):
        layers = O.mmcs_commit(O.hasher(O.GOLDILOCKS, bench.P2_SEED, p2w), [lde])
        out[f"root_w{p2w}"] = [str(int(x)) for x in layers[-1][0]]
        del layers
    print(f"goldilocks: {time.time() - t0:.0f} s", flush=True)
    return out


def main() -> None:
    O.build()
    res = {"generator": "tests/golden/make_fullsize.py (oracle/ C restatement)",
           "babybear_2^22x256_b2": babybear_headline(),
           "goldilocks_2^20x64_b4": goldilocks_lde()}
    with open(OUT, "w") as f:
        json.dump(res, f, indent=1)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
