"""The continuous-batching engine: results are identical alone and in the mix.

Jobs of mixed sizes (both fields, with and without the FRI phase) run first one at a
time on a one-slot engine, then all submitted at once to a four-slot engine where they
overlap on the GPU; every root, FRI commitment, final codeword and query answer must
match bit for bit (tolerance 0), and match the oracle for the small ones."""
import numpy as np
import pytest

import ziros_b200 as Z
from conftest import rand_field

pytestmark = pytest.mark.gpu


def _jobs():
    jobs = []
    for k, (field, log_h, w) in enumerate([(0, 12, 16), (0, 14, 40), (1, 10, 24), (0, 16, 64), (0, 9, 8),
                                           (1, 13, 8), (0, 15, 128), (0, 11, 256)]):
        trace = rand_field(field, (1 << log_h, w), 900 + k)
        fri = None
        if field == 0 and k % 2 == 0:
            fri = {"alpha": rand_field(0, 4, 950 + k), "log_final": 3, "num_queries": 7,
                   "challenge_seed": 17 + k, "query_seed": 23 + k}
        jobs.append((field, trace, fri))
    return jobs


def _run(engine, jobs, concurrent):
    out = [None] * len(jobs)
    if concurrent:
        ids = [engine.submit(t, field=f, seed=42, log_blowup=1, fri=fr) for f, t, fr in jobs]
        for i, jid in enumerate(ids):
            out[i] = engine.wait(jid)
    else:
        for i, (f, t, fr) in enumerate(jobs):
            out[i] = engine.wait(engine.submit(t, field=f, seed=42, log_blowup=1, fri=fr))
    return out


def test_results_identical_alone_and_in_the_mix(oracle):
    jobs = _jobs()
    solo = Z.CommitEngine(slots=1)
    alone = _run(solo, jobs, concurrent=False)
    solo.close()
    eng = Z.CommitEngine(slots=4)
    mixed = _run(eng, jobs, concurrent=True)
    st = eng.stats()
    eng.close()
    assert st["completed"] == len(jobs) and st["hbm_peak"] <= st["hbm_budget"]
    for (field, trace, fri), a, m in zip(jobs, alone, mixed):
        assert (a[0] == m[0]).all()
        if fri:
            assert (a[1].roots == m[1].roots).all() and (a[1].final == m[1].final).all()
            assert (a[1].query_rows == m[1].query_rows).all()
            assert (a[1].query_siblings == m[1].query_siblings).all()
        else:
            assert a[1] is None and m[1] is None
    # small jobs against the oracle
    for (field, trace, fri), a in zip(jobs, alone):
        if trace.shape[0] <= 1 << 12:
            lde = oracle.coset_lde(field, trace, 1)
            layers = oracle.mmcs_commit(oracle.hasher(field, 42), [lde])
            assert (a[0] == layers[-1][0]).all()


def test_admission_by_hbm_budget():
    """A budget that fits one job at a time still completes every job correctly."""
    jobs = [(0, rand_field(0, (1 << 14, 32), 60 + k), None) for k in range(4)]
    ref = Z.CommitEngine(slots=1)
    want = _run(ref, jobs, concurrent=False)
    ref.close()
    per_job = (1 << 14) * 32 * 4 * 4 + (64 << 20)
    eng = Z.CommitEngine(slots=4, hbm_budget=int(per_job * 1.5))
    got = _run(eng, jobs, concurrent=True)
    st = eng.stats()
    eng.close()
    assert st["hbm_peak"] <= st["hbm_budget"]
    for a, b in zip(want, got):
        assert (a[0] == b[0]).all()


def test_rejects_job_larger_than_budget():
    eng = Z.CommitEngine(slots=1, hbm_budget=1 << 20)
    with pytest.raises(Z.ZkbError):
        eng.submit(rand_field(0, (1 << 12, 16), 1))
    eng.close()


def test_job_log_lines_and_nvtx_ranges(tmp_path):
    """ZKB_JOB_LOG writes one JSON line per finished job; ZKB_NVTX=1 wraps launches in
    NVTX ranges (checked here only for not disturbing the results).  Both are read once
    per process, so the check runs in a fresh one."""
    import json
    import os
    import subprocess
    import sys

    log = tmp_path / "jobs.jsonl"
    code = ("import numpy as np, ziros_b200 as Z\n"
            "rng = np.random.default_rng(1)\n"
            "e = Z.CommitEngine(slots=2)\n"
            "ids = [e.submit(rng.integers(0, 0x78000001, size=(1 << h, w), dtype=np.uint32))"
            " for h, w in ((10, 16), (12, 24))]\n"
            "roots = [e.wait(i)[0] for i in ids]\n"
            "e.close()\n"
            "print(' '.join(str(int(r[0])) for r in roots))\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], env=dict(os.environ, ZKB_JOB_LOG=str(log), ZKB_NVTX="1"),
                         capture_output=True, text=True, timeout=300, cwd=root)
    assert out.returncode == 0, out.stderr
    lines = [json.loads(x) for x in log.read_text().splitlines()]
    assert sorted((d["log_h"], d["width"]) for d in lines) == [(10, 16), (12, 24)]
    assert all(d["status"] == 0 and d["latency_ms"] >= d["run_ms"] >= 0 for d in lines)


def test_smallest_policy_results_identical_to_alone():
    jobs = _jobs()
    solo = Z.CommitEngine(slots=1)
    alone = _run(solo, jobs, concurrent=False)
    solo.close()
    eng = Z.CommitEngine(slots=3, policy="smallest")
    mixed = _run(eng, jobs, concurrent=True)
    eng.close()
    for (field, trace, fri), a, m in zip(jobs, alone, mixed):
        assert (a[0] == m[0]).all()
        if fri:
            assert (a[1].roots == m[1].roots).all() and (a[1].query_siblings == m[1].query_siblings).all()


def _start_order(policy, n_small):
    """One slot: a long job runs while a medium job and then n_small small jobs queue up;
    returns the labels in the order the jobs started."""
    import time

    big = rand_field(0, (1 << 19, 64), 70)
    medium = rand_field(0, (1 << 16, 32), 71)
    smalls = [rand_field(0, (1 << 10, 8), 72 + k) for k in range(n_small)]
    eng = Z.CommitEngine(slots=1, policy=policy)
    subs = []
    for label, t in [("big", big), ("medium", medium)] + [(f"small{k}", s) for k, s in enumerate(smalls)]:
        jid = eng.submit(t, field=0, seed=42, log_blowup=1)
        subs.append((label, jid, time.perf_counter()))
        if label == "big":  # the slot takes it before anything else is queued
            t0 = time.perf_counter()
            while eng.stats()["queued"] and time.perf_counter() - t0 < 10:
                time.sleep(0.0002)
    starts = []
    for label, jid, t_sub in subs:
        res = eng.wait(jid)
        starts.append((t_sub + res[2]["queue_ms"] / 1e3, label))
    eng.close()
    return [label for _, label in sorted(starts)]


def test_fifo_admits_in_arrival_order():
    order = _start_order("fifo", 3)
    assert order == ["big", "medium", "small0", "small1", "small2"]


def test_smallest_first_with_bounded_bypass():
    """The small jobs pass the medium one until it has been passed over
    ZKB_ADMIT_MAX_BYPASS times; then it goes next."""
    from ziros_b200 import _native as N

    order = _start_order("smallest", N.ADMIT_MAX_BYPASS + 2)
    assert order[0] == "big"
    assert order.index("medium") == 1 + N.ADMIT_MAX_BYPASS
    assert all(x.startswith("small") for x in order[1:1 + N.ADMIT_MAX_BYPASS])


def test_unknown_policy_is_rejected():
    with pytest.raises(ValueError):
        Z.CommitEngine(slots=1, policy="lifo")


def test_fifo_backfill_passes_a_waiting_job_a_bounded_number_of_times():
    """FIFO with a budget that holds the big job and one small one but not the medium one:
    small jobs backfill past the waiting medium job at most ZKB_ADMIT_MAX_BYPASS times."""
    import time

    from ziros_b200 import _native as N

    MiB = 1 << 20
    est = lambda log_h, w: (1 << log_h) * w * 4 + (2 << log_h) * w * 4 + 2 * (2 << log_h) * 64 + 64 * MiB
    big_shape, med_shape, small_shape = (20, 64), (16, 32), (10, 8)
    budget = est(*big_shape) + est(*small_shape) + 8 * MiB
    assert est(*big_shape) + est(*med_shape) > budget
    big = rand_field(0, (1 << big_shape[0], big_shape[1]), 80)
    medium = rand_field(0, (1 << med_shape[0], med_shape[1]), 81)
    smalls = [rand_field(0, (1 << small_shape[0], small_shape[1]), 82 + k) for k in range(N.ADMIT_MAX_BYPASS + 3)]
    eng = Z.CommitEngine(slots=2, hbm_budget=budget, policy="fifo")
    subs = []
    for label, t in [("big", big), ("medium", medium)] + [(f"small{k}", s) for k, s in enumerate(smalls)]:
        jid = eng.submit(t, field=0, seed=42, log_blowup=1)
        subs.append((label, jid, time.perf_counter()))
        if label == "big":
            t0 = time.perf_counter()
            while eng.stats()["queued"] and time.perf_counter() - t0 < 10:
                time.sleep(0.0002)
    starts = []
    for label, jid, t_sub in subs:
        res = eng.wait(jid)
        starts.append((t_sub + res[2]["queue_ms"] / 1e3, label))
    st = eng.stats()
    eng.close()
    order = [label for _, label in sorted(starts)]
    assert order[0] == "big"
    assert order.index("medium") <= 1 + N.ADMIT_MAX_BYPASS
    assert st["hbm_peak"] <= budget
