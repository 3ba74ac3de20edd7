"""Host traces uploaded a column slab at a time (BabyBear, width-16 hasher, width >= 128):
every slab's LDE and leaf absorption start once it has landed.  The commitment must equal
the device-resident path's (no slabs) bit for bit — root, every opening, the FRI
commitments, final codeword and query answers — for widths that end in a full slab, in a
slab of a few columns, and in a partial absorbed chunk, through the plain host call and
through the engine."""
import numpy as np
import pytest
import torch

import ziros_b200 as Z
from conftest import rand_field

pytestmark = pytest.mark.gpu

WIDTHS = [128, 136, 130, 200, 257, 512]


def _dev(t):
    return torch.from_numpy(np.ascontiguousarray(t).view(np.int32)).cuda()


@pytest.mark.parametrize("width", WIDTHS)
@pytest.mark.parametrize("log_h", [1, 6, 13])
def test_host_commit_equals_device_commit(width, log_h):
    t = rand_field(Z.BABYBEAR, (1 << log_h, width), 3000 + width + log_h)
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    root_h, tree_h = pcs.commit(t)
    root_d, tree_d = pcs.commit_dev(_dev(t))
    assert (root_h == root_d).all()
    n = 2 << log_h
    for idx in (0, n - 1, n // 3):
        a = pcs.mmcs.open_batch(idx, tree_h)
        b = pcs.mmcs.open_batch(idx, tree_d)
        assert all((x == y).all() for x, y in zip(a[0], b[0]))
        assert all((x == y).all() for x, y in zip(a[1], b[1]))


def _same_proof(p, q):
    assert (p.roots == q.roots).all() and (p.betas == q.betas).all()
    assert (p.final == q.final).all()
    assert (p.query_indices == q.query_indices).all()
    assert (p.query_rows == q.query_rows).all() and (p.query_siblings == q.query_siblings).all()


@pytest.mark.parametrize("width,transcript", [(136, False), (257, False), (200, True)])
def test_host_commit_fri_equals_device(width, transcript):
    t = rand_field(Z.BABYBEAR, (1 << 12, width), 3100 + width)
    alpha = rand_field(Z.BABYBEAR, 4, 3150)
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    kw = dict(log_final=4, num_queries=9, challenge_seed=5, query_seed=6, transcript=transcript)
    r_h, _, p_h = pcs.commit_fri(t, alpha, want_tree=False, **kw)
    r_d, _, p_d = pcs.commit_fri_dev(_dev(t), alpha, **kw)
    assert (r_h == r_d).all()
    _same_proof(p_h, p_d)


def test_engine_slabbed_jobs_equal_device_path():
    shapes = [(1 << 13, 256), (1 << 11, 136), (1 << 12, 130), (1 << 10, 64)]
    fri = {"alpha": [11, 22, 33, 44], "log_final": 3, "num_queries": 5, "challenge_seed": 3, "query_seed": 4}
    traces = [rand_field(Z.BABYBEAR, s, 3200 + i) for i, s in enumerate(shapes)]
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    want = [pcs.commit_fri_dev(_dev(t), fri["alpha"], fri["log_final"], fri["num_queries"], fri["challenge_seed"],
                               fri["query_seed"]) for t in traces]
    eng = Z.CommitEngine(slots=3)
    try:
        ids = [eng.submit(t, field=Z.BABYBEAR, seed=42, log_blowup=1, fri=fri) for t in traces]
        for (root, _, pf), jid in zip(want, ids):
            r, p, _ = eng.wait(jid)
            assert (r == root).all()
            _same_proof(p, pf)
    finally:
        eng.close()


def test_pinned_host_commit_equals_device_commit():
    t = rand_field(Z.BABYBEAR, (1 << 14, 192), 3300)
    pinned = torch.from_numpy(t.view(np.int32)).pin_memory()
    pcs = Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1)
    root_p, _ = pcs.commit_ptr(pinned.data_ptr(), 1 << 14, 192, want_tree=False)
    root_d, _ = pcs.commit_dev(_dev(t), want_tree=False)
    assert (root_p == root_d).all()
