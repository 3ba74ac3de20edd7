"""The persistent form of the batched commit: one kernel fed by a device work queue.

Every root must equal that trace's plain commitment (CudaTwoAdicPcs.commit, itself pinned
to the oracle) for any Merkle-level fusion, blowup and mix of shapes (tiny traces whose
passes are one bit, traces of one 256-row leaf tile, uneven widths); openings through the
plan's trees equal the plain tree's; the autotuner's choice is cached; and a work item
whose dependency never completes makes the kernel give up after its spin limit and report
ZKB_ERR_TIMEOUT (the wait is bounded; the GPU is not faulted), after which the plan runs
correctly again."""
import numpy as np
import pytest

import ziros_b200 as Z
from conftest import rand_field
from ziros_b200 import _native as N

pytestmark = pytest.mark.gpu

# widths multiples of 8; heights 2^1 .. 2^14 (one-bit passes, fused-only plans, plans of
# three passes), and 2^7 rows so the LDE is one leaf tile
SHAPES = [(1 << 12, 256), (1 << 1, 8), (1 << 9, 16), (1 << 14, 24), (1 << 7, 40), (1 << 3, 8), (1 << 11, 136),
          (1 << 13, 8), (1 << 10, 64), (1 << 5, 72)]


def _run(shapes, traces, **kw):
    b = Z.BatchCommit(shapes, persistent=True, **kw)
    for i, t in enumerate(traces):
        b.copy_in(i, t)
    b.run()
    return b, b.roots()


def _plain(traces, log_blowup=1):
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, log_blowup)
    return [pcs.commit(t)[0] for t in traces]


@pytest.mark.parametrize("log_blowup", [1, 2])
def test_persistent_roots_equal_plain_commits(log_blowup):
    traces = [rand_field(Z.BABYBEAR, s, 1200 + i) for i, s in enumerate(SHAPES)]
    want = _plain(traces, log_blowup)
    b, got = _run(SHAPES, traces, log_blowup=log_blowup, autotune=False)
    for i in range(len(SHAPES)):
        assert (got[i] == want[i]).all(), f"trace {i} shape {SHAPES[i]}"
    info, q = b.info(), b.queue_info()
    assert info["use_graph"] == 2 and info["kernels_per_run"] == 1
    assert q["items"] > 0 and q["steps"] >= 3 * len(SHAPES) and q["grid"] > 0


@pytest.mark.parametrize("slots", [1, 3])
def test_shared_coefficient_scratch(monkeypatch, slots):
    """Traces share S scratch slots round-robin (largest first); each waits for the previous
    user's fused step.  One and three slots for ten traces: the same roots."""
    monkeypatch.setenv("ZKB_PERSIST_SLOTS", str(slots))
    traces = [rand_field(Z.BABYBEAR, s, 1250 + i) for i, s in enumerate(SHAPES)]
    want = _plain(traces)
    b, got = _run(SHAPES, traces, autotune=False)
    for i in range(len(SHAPES)):
        assert (got[i] == want[i]).all(), f"trace {i} shape {SHAPES[i]} slots {slots}"
    b.set_merkle_fusion(4, 3)
    b.run()
    assert all((g == w).all() for g, w in zip(b.roots(), want))


@pytest.mark.parametrize("leaf_levels,comp_levels", [(0, 1), (8, 8), (3, 4), (1, 2), (5, 7)])
def test_every_merkle_fusion_gives_the_same_roots(leaf_levels, comp_levels):
    traces = [rand_field(Z.BABYBEAR, s, 1300 + i) for i, s in enumerate(SHAPES)]
    want = _plain(traces)
    b, _ = _run(SHAPES, traces, autotune=False)
    b.set_merkle_fusion(leaf_levels, comp_levels)
    b.run()
    got = b.roots()
    assert b.queue_info()["leaf_levels"] == leaf_levels
    for i in range(len(SHAPES)):
        assert (got[i] == want[i]).all(), f"trace {i} fusion ({leaf_levels}, {comp_levels})"
    # every digest layer, not only the root
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    for i in (0, 3, 4):
        _, tree = pcs.commit(traces[i])
        bt = b.tree(i)
        for lvl in range(tree.num_layers()):
            assert (bt.layer(lvl) == tree.layer(lvl)).all(), f"trace {i} layer {lvl}"


def test_openings_through_persistent_trees():
    traces = [rand_field(Z.BABYBEAR, s, 1400 + i) for i, s in enumerate(SHAPES)]
    b, _ = _run(SHAPES, traces, autotune=False)
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    mmcs = Z.CudaMerkleTreeMmcs(Z.BABYBEAR, 42)
    for i in (0, 2, 6):
        _, tree = pcs.commit(traces[i])
        rows = SHAPES[i][0] * 2
        for idx in (0, rows // 3, rows - 1):
            got_rows, got_proof = mmcs.open_batch(idx, b.tree(i))
            want_rows, want_proof = mmcs.open_batch(idx, tree)
            assert all((a == c).all() for a, c in zip(got_rows, want_rows))
            assert all((a == c).all() for a, c in zip(got_proof, want_proof))


def test_autotuned_fusion_is_cached(tmp_path):
    shapes = SHAPES[:6]
    traces = [rand_field(Z.BABYBEAR, s, 1500 + i) for i, s in enumerate(shapes)]
    want = _plain(traces)
    cache = str(tmp_path / "tune.jsonl")
    b, got = _run(shapes, traces, autotune=True, tune_cache=cache)
    assert all((g == w).all() for g, w in zip(got, want))
    chosen = b.queue_info()
    assert '"leaf_levels"' in open(cache).read()
    b2, got2 = _run(shapes, traces, autotune=True, tune_cache=cache)
    assert b2.info()["tuned_from_cache"] == 1
    q2 = b2.queue_info()
    assert (q2["leaf_levels"], q2["comp_levels"]) == (chosen["leaf_levels"], chosen["comp_levels"])
    assert all((g == w).all() for g, w in zip(got2, want))


def test_a_dependency_that_never_completes_times_out_and_the_plan_recovers():
    traces = [rand_field(Z.BABYBEAR, s, 1600 + i) for i, s in enumerate(SHAPES)]
    want = _plain(traces)
    b, _ = _run(SHAPES, traces, autotune=False)
    b.debug_stalled_run(spin_limit=2000)
    with pytest.raises(Z.ZkbError) as e:
        b.roots()
    assert e.value.code == N.ERR_TIMEOUT and "spin limit" in str(e.value)
    assert N.circuit_open()[0] is False  # a bounded wait, not a device failure
    b.run()
    got = b.roots()
    assert all((g == w).all() for g, w in zip(got, want))


def test_persistent_form_rejects_unsupported_shapes():
    with pytest.raises(Z.ZkbError):
        Z.BatchCommit([(1 << 4, 7)], persistent=True, autotune=False)
    with pytest.raises(Z.ZkbError):
        Z.BatchCommit([(1 << 4, 8)], field=Z.GOLDILOCKS, persistent=True, autotune=False)
