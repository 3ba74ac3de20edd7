"""The full-size fixtures and the seeded trace they answer for (CPU).

tests/golden/fullsize.json holds the oracle's answers for traces drawn by
bench.synthetic_trace; these tests pin that generator's stream (a prefix of a large
draw equals a small draw, and the first values are fixed), so the GPU tests and
bench.py regenerate exactly the traces the fixtures were made from, and check that
the fixture file is complete."""
import json
import os

import bench

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fullsize.json")


def test_synthetic_trace_stream_is_pinned():
    a = bench.synthetic_trace(0, 4, 4, bench.TRACE_SEED)
    assert a.tolist()[0] == [1277659838, 269326308, 1348838822, 824033045]
    assert a.tolist()[3] == [1730030357, 604943717, 1897644294, 897556106]
    b = bench.synthetic_trace(1, 2, 2, bench.TRACE_SEED)
    assert [int(x) for x in b[1]] == [8838455141052702686, 15748455042934720403]
    big = bench.synthetic_trace(0, 1 << 12, 4096, bench.TRACE_SEED)  # spans block boundaries
    assert big.reshape(-1)[:16].tolist() == a.reshape(-1).tolist()
    assert int(big.max()) < bench.BB_P and int(b.max()) < bench.GL_P


def test_fullsize_fixture_is_complete():
    with open(GOLDEN) as f:
        g = json.load(f)
    bb = g["babybear_2^22x256_b2"]
    wl = bench.WORKLOADS["babybear_2^22x256_b2"]
    assert (bb["log_rows"], bb["width"], bb["log_blowup"]) == (wl["log_h"], wl["width"], wl["log_blowup"])
    assert bb["trace_seed"] == bench.TRACE_SEED and bb["alpha"] == list(bench.ALPHA) and bb["fri"] == bench.FRI
    rounds = wl["log_h"] + wl["log_blowup"] - bench.FRI["log_final"]
    assert len(bb["fri_roots"]) == len(bb["fri_betas"]) == rounds
    assert len(bb["fri_final"]) == 1 << bench.FRI["log_final"]
    assert len(bb["query_indices"]) == bench.FRI["num_queries"] and len(bb["root"]) == 8
    gl = g["goldilocks_2^20x64_b4"]
    assert len(gl["lde_block_sha256"]) == (1 << (gl["log_rows"] + gl["log_blowup"])) // gl["block_rows"]
    assert len(gl["root_w16"]) == 8 and len(gl["root_w12"]) == 4
