"""Batched commit (one plan, one CUDA graph per run) against the plain per-trace path.

Every root of a batch must equal that trace's plain commitment (CudaTwoAdicPcs.commit,
itself pinned to the oracle), bit for bit, whatever kernel shapes the autotuner picks,
with and without the graph, for any branch count; openings through the batch's trees
equal the plain tree's."""
import numpy as np
import pytest

import ziros_b200 as Z
from conftest import rand_field

pytestmark = pytest.mark.gpu

MIXED = [(1 << 3, 7), (1 << 9, 8), (1 << 12, 256), (1 << 13, 40), (1 << 10, 16), (1 << 1, 1), (1 << 14, 24),
         (1 << 12, 8), (1 << 0, 5), (1 << 11, 128)]


def _traces(field, shapes, seed):
    return [rand_field(field, s, seed + i) for i, s in enumerate(shapes)]


def _plain_roots(field, traces, log_blowup=1, p2w=16):
    pcs = Z.CudaTwoAdicPcs(field, 42, log_blowup, p2w)
    return [pcs.commit(t)[0] for t in traces]


def _batch_roots(field, shapes, traces, **kw):
    b = Z.BatchCommit(shapes, field=field, **kw)
    for i, t in enumerate(traces):
        b.copy_in(i, t)
    b.run()
    return b, b.roots()


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_roots_equal_plain_commits(tmp_path, use_graph):
    traces = _traces(Z.BABYBEAR, MIXED, 700)
    want = _plain_roots(Z.BABYBEAR, traces)
    b, got = _batch_roots(Z.BABYBEAR, MIXED, traces, use_graph=use_graph, autotune=True,
                          tune_cache=str(tmp_path / "tune.jsonl"))
    for i in range(len(MIXED)):
        assert (got[i] == want[i]).all(), f"trace {i} shape {MIXED[i]}"
    info = b.info()
    assert info["use_graph"] == int(use_graph) and info["device_bytes"] > 0
    if use_graph:
        assert info["kernels_per_run"] > 0


def test_small_batch_against_oracle(oracle):
    shapes = [(1 << 4, 8), (1 << 6, 3), (1 << 2, 17)]
    traces = _traces(Z.BABYBEAR, shapes, 5)
    _, got = _batch_roots(Z.BABYBEAR, shapes, traces, autotune=False)
    h = oracle.hasher(Z.BABYBEAR, 42)
    for t, r in zip(traces, got):
        lde = oracle.coset_lde(Z.BABYBEAR, t, 1)
        assert (r == oracle.mmcs_commit(h, [lde])[-1][0]).all()


@pytest.mark.parametrize("branches", [1, 3, 8])
def test_branch_counts_agree(branches):
    traces = _traces(Z.BABYBEAR, MIXED, 800)
    want = _plain_roots(Z.BABYBEAR, traces)
    _, got = _batch_roots(Z.BABYBEAR, MIXED, traces, autotune=False, branches=branches)
    assert all((g == w).all() for g, w in zip(got, want))


@pytest.mark.parametrize("p2w", [16, 12])
def test_goldilocks_batch(p2w):
    shapes = [(1 << 10, 64), (1 << 7, 8), (1 << 12, 12), (1 << 3, 1)]
    traces = _traces(Z.GOLDILOCKS, shapes, 900)
    want = _plain_roots(Z.GOLDILOCKS, traces, log_blowup=2, p2w=p2w)
    _, got = _batch_roots(Z.GOLDILOCKS, shapes, traces, log_blowup=2, p2_width=p2w, autotune=True)
    assert all((g == w).all() for g, w in zip(got, want))


def test_openings_through_batch_trees():
    traces = _traces(Z.BABYBEAR, MIXED, 1000)
    b, _ = _batch_roots(Z.BABYBEAR, MIXED, traces, autotune=False)
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    for i in (2, 3, 5, 8):
        _, plain_tree = pcs.commit(traces[i])
        n = MIXED[i][0] << 1
        for idx in (0, n - 1, n // 3):
            got = pcs.mmcs.open_batch(idx, b.tree(i))
            want = pcs.mmcs.open_batch(idx, plain_tree)
            assert all((x == y).all() for x, y in zip(got[0], want[0]))
            assert all((x == y).all() for x, y in zip(got[1], want[1]))


def test_rerun_with_new_traces():
    shapes = MIXED[:6]
    b = Z.BatchCommit(shapes, autotune=False)
    for rep in range(2):
        traces = _traces(Z.BABYBEAR, shapes, 1100 + 50 * rep)
        for i, t in enumerate(traces):
            b.copy_in(i, t)
        b.run()
        got = b.roots()
        want = _plain_roots(Z.BABYBEAR, traces)
        assert all((g == w).all() for g, w in zip(got, want))


def test_device_sources_and_replay():
    import torch

    shapes = [(1 << 12, 32), (1 << 9, 8)]
    traces = _traces(Z.BABYBEAR, shapes, 1200)
    b = Z.BatchCommit(shapes, autotune=False)
    dev = [torch.from_numpy(t.view(np.int32)).cuda() for t in traces]
    for i, t in enumerate(dev):
        b.copy_in(i, t)
    for _ in range(3):
        b.run()
    got = b.roots()
    want = _plain_roots(Z.BABYBEAR, traces)
    assert all((g == w).all() for g, w in zip(got, want))


def test_tune_cache_roundtrip(tmp_path):
    path = str(tmp_path / "tune.jsonl")
    shapes = [(1 << 13, 64), (1 << 15, 16), (1 << 12, 8)]
    a = Z.BatchCommit(shapes, autotune=True, tune_cache=path)
    tunes = [a.lde_tune(i) for i in range(len(shapes))]
    info_a = a.info()
    a.close()
    lines = open(path).read().strip().splitlines()
    assert any('"key": "lde/0/13/64/1"' in ln for ln in lines)
    assert any('"key": "branches/' in ln for ln in lines)
    b = Z.BatchCommit(shapes, autotune=False, tune_cache=path)
    assert b.info()["tuned_from_cache"] == 1
    assert [b.lde_tune(i) for i in range(len(shapes))] == tunes
    assert b.info()["branches"] == info_a["branches"] and b.info()["leaf_threads"] == info_a["leaf_threads"]


@pytest.mark.parametrize("field,log_h,width", [(Z.BABYBEAR, 14, 48), (Z.BABYBEAR, 20, 16), (Z.GOLDILOCKS, 13, 24),
                                               (Z.BABYBEAR, 9, 7), (Z.BABYBEAR, 12, 415), (Z.GOLDILOCKS, 11, 29)])
def test_every_lde_kernel_shape_gives_the_same_lde(field, log_h, width):
    """The autotuner's candidates (pass split, column chunks) are all the same function."""
    import torch

    trace = rand_field(field, (1 << log_h, width), 1300 + log_h)
    tt = torch.from_numpy(trace.view(np.int32 if field == Z.BABYBEAR else np.int64)).cuda()
    dft = Z.CudaDft(field)
    ref = torch.empty((2 << log_h, width), dtype=tt.dtype, device="cuda")
    dft.coset_lde_batch_dev(tt, 1, ref)
    kdef = 11 if field == Z.BABYBEAR else 10
    for kmax in (kdef, kdef - 1, kdef - 2, 5, 3):
        for cp in (16, 8, 4, 1):
            for cf in (8, 4, 1):
                if field == Z.GOLDILOCKS and cp == 16:
                    continue
                out = torch.empty_like(ref)
                dft.coset_lde_tuned_dev(tt, 1, out, kmax, cp, cf)
                torch.cuda.synchronize()
                assert torch.equal(out, ref), (kmax, cp, cf)


def test_rejects_bad_shapes():
    with pytest.raises(Z.ZkbError):
        Z.BatchCommit([(1 << 27, 8)])
    with pytest.raises(Z.ZkbError):
        Z.BatchCommit([(1 << 4, 0)])
    with pytest.raises(ValueError):
        Z.BatchCommit([(24, 8)])


def test_config4_shape_distribution_at_reduced_height():
    """64 uneven traces (log2 rows uniform in [4, 14], widths uniform in {8, ..., 256}):
    the same draw as the batched workload at a smaller height range."""
    rng = np.random.default_rng(4)
    shapes = [(1 << int(rng.integers(4, 15)), 8 * int(rng.integers(1, 33))) for _ in range(64)]
    traces = _traces(Z.BABYBEAR, shapes, 2000)
    want = _plain_roots(Z.BABYBEAR, traces)
    _, got = _batch_roots(Z.BABYBEAR, shapes, traces, autotune=True)
    assert all((g == w).all() for g, w in zip(got, want))


# ---- runs from host memory (zkb_batch_run_host): copies overlapped with the commitment,
# traces committed in groups (smallest first) as their copies land


@pytest.mark.parametrize("branches,use_graph", [(1, True), (3, True), (2, False)])
def test_run_host_roots_equal_plain_commits(branches, use_graph):
    b = Z.BatchCommit(MIXED, autotune=False, branches=branches, use_graph=use_graph)
    for rep in range(2):
        traces = _traces(Z.BABYBEAR, MIXED, 1300 + 40 * rep)
        b.run_host(traces)
        got = b.roots()
        want = _plain_roots(Z.BABYBEAR, traces)
        for i in range(len(MIXED)):
            assert (got[i] == want[i]).all(), f"rep {rep} trace {i} shape {MIXED[i]}"


def test_run_host_pinned_sources_alternating_with_graph_runs():
    import torch

    shapes = MIXED[:7]
    b = Z.BatchCommit(shapes, autotune=False)
    for rep in range(3):
        traces = _traces(Z.BABYBEAR, shapes, 1400 + 30 * rep)
        want = _plain_roots(Z.BABYBEAR, traces)
        pinned = [torch.from_numpy(t.view(np.int32)).pin_memory() for t in traces]
        b.run_host(pinned)
        got = b.roots()
        assert all((g == w).all() for g, w in zip(got, want)), f"rep {rep} run_host"
        # the graph form on the same plan after a host run, with other traces
        other = _traces(Z.BABYBEAR, shapes, 1500 + 30 * rep)
        for i, t in enumerate(other):
            b.copy_in(i, t)
        b.run()
        got = b.roots()
        want2 = _plain_roots(Z.BABYBEAR, other)
        assert all((g == w).all() for g, w in zip(got, want2)), f"rep {rep} graph run"


@pytest.mark.parametrize("p2w", [16, 12])
def test_run_host_goldilocks(p2w):
    shapes = [(1 << 10, 64), (1 << 7, 8), (1 << 12, 12), (1 << 3, 1)]
    traces = _traces(Z.GOLDILOCKS, shapes, 1600)
    want = _plain_roots(Z.GOLDILOCKS, traces, log_blowup=2, p2w=p2w)
    b = Z.BatchCommit(shapes, field=Z.GOLDILOCKS, log_blowup=2, p2_width=p2w, autotune=False, branches=2)
    b.run_host(traces)
    assert all((g == w).all() for g, w in zip(b.roots(), want))


def test_run_host_persistent_plan():
    shapes = [(1 << 12, 16), (1 << 9, 8), (1 << 14, 24), (1 << 6, 64)]
    traces = _traces(Z.BABYBEAR, shapes, 1700)
    want = _plain_roots(Z.BABYBEAR, traces)
    b = Z.BatchCommit(shapes, persistent=True, autotune=False)
    b.run_host(traces)
    assert all((g == w).all() for g, w in zip(b.roots(), want))


def test_openings_after_run_host():
    traces = _traces(Z.BABYBEAR, MIXED, 1800)
    b = Z.BatchCommit(MIXED, autotune=False, branches=2)
    b.run_host(traces)
    b.roots()
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    for i in (2, 6, 9):
        _, plain_tree = pcs.commit(traces[i])
        n = MIXED[i][0] << 1
        for idx in (0, n - 1, n // 5):
            got = pcs.mmcs.open_batch(idx, b.tree(i))
            want = pcs.mmcs.open_batch(idx, plain_tree)
            assert all((x == y).all() for x, y in zip(got[0], want[0]))
            assert all((x == y).all() for x, y in zip(got[1], want[1]))


def test_run_host_rejects_bad_sources():
    import torch

    shapes = [(1 << 4, 8), (1 << 5, 3)]
    b = Z.BatchCommit(shapes, autotune=False)
    traces = _traces(Z.BABYBEAR, shapes, 1900)
    with pytest.raises(ValueError):
        b.run_host(traces[:1])
    with pytest.raises(ValueError):
        b.run_host([traces[1], traces[0]])
    with pytest.raises(ValueError):
        b.run_host([torch.from_numpy(traces[0].view(np.int32)).cuda(), traces[1]])


def test_run_host_many_groups():
    # 40 traces of growing size: the smallest share groups, the largest stand alone
    shapes = [(1 << (4 + i % 9), 8 + 8 * (i % 5)) for i in range(40)]
    traces = _traces(Z.BABYBEAR, shapes, 2000)
    want = _plain_roots(Z.BABYBEAR, traces)
    b = Z.BatchCommit(shapes, autotune=False, branches=4)
    b.run_host(traces)
    got = b.roots()
    for i in range(len(shapes)):
        assert (got[i] == want[i]).all(), f"trace {i} shape {shapes[i]}"
