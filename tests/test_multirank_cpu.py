"""The N > 1 host path of bench.py on CPU: world_size-2 gloo process groups.

Replicas exchange nothing but the barrier and the max over ranks of the timed region;
rank 0 alone reports.  These tests run the same Ranks helper the GPU runs use (with
gloo instead of NCCL), in spawned processes."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    r = bench.Ranks(world, torch.device("cpu"), backend="gloo", timeout_s=60)
    local = 1.5 + rank  # each rank's own timed region
    r.barrier()
    t_max = r.max(local)
    value = bench.whole_job_rate(1000.0, 4, world, t_max)
    r.barrier()
    r.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"t_max": t_max, "value": value}, f)


def test_two_rank_max_and_whole_job_rate(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    # every rank sees the slowest rank's time; the rate counts every rank's units
    assert all(r["t_max"] == pytest.approx(2.5) for r in res)
    assert all(r["value"] == pytest.approx(1000.0 * 4 * 2 / 2.5) for r in res)


def test_single_rank_needs_no_process_group():
    r = bench.Ranks(1, torch.device("cpu"), backend="gloo")
    assert r.dist is None and r.max(3.0) == 3.0
    r.barrier()
    r.close()


def test_reference_arm_prints_only_on_rank_zero():
    class Args:
        steps, warmup, workload = 1, 0, "babybear_2^14x16_b2"

    buf = io.StringIO()
    with redirect_stdout(buf):
        rc = bench.run_reference(Args(), bench.WORKLOADS[Args.workload], rank=1, world=2)
    assert rc == 0 and buf.getvalue() == ""


def test_workloads_have_a_metric_and_valid_shapes():
    for name, wl in bench.WORKLOADS.items():
        assert wl["field"] in (0, 1) and wl["log_blowup"] >= 1, name
    shapes = bench.batch_shapes(bench.WORKLOADS["batch64_babybear"])
    assert len(shapes) == 64 and all(12 <= h.bit_length() - 1 <= 22 and w % 8 == 0 and 8 <= w <= 256
                                      for h, w in shapes)
    jobs = bench.serving_jobs(bench.WORKLOADS["serving_babybear"], 60, 5)
    assert all(14 <= h.bit_length() - 1 <= 24 and 32 <= w <= 512 for h, w in jobs)
