#!/usr/bin/env python
"""Benchmark of the polynomial-commitment hot path: trace cells/s committed.

One step is one commitment job on a synthetic trace (zkb_pcs_commit_fri): coset LDE
(blowup 2^log_blowup, shift = field generator) with rows bit-reversed, Poseidon2
MMCS over the rows (TwoAdicFriPcs::commit), then for BabyBear the alpha-reduction of
the committed columns into one F_p^4 codeword and the FRI commit phase on it (fold by
2 down to 2^8 with a Merkle commit per layer, 100 query openings).  The default
workload is BabyBear 2^22 rows x 256 columns, blowup 2 — the 2^22 x 256 BabyBear
LDE+commit named as the target shape; `--workload` selects the others (Goldilocks
jobs commit without the extension FRI phase).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value : whole-job cells/s with the trace resident in HBM (CUDA events on the
        launching stream, max over ranks).
e2e   : the same metric through the serving engine (zkb_engine_submit/wait, four
        slots) with the trace in pinned host memory: every job's H2D copy and the
        D2H read of its root and FRI answers are inside the timed region; one job's
        copy overlaps another's kernels.
--impl reference : the reference CPU path (restated in C, oracle/) on the host
        cores, on a bounded sample of the same workload.
N > 1 runs one independent replica per GPU (torchrun; no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BB_P = 0x78000001
GL_P = 0xFFFFFFFF00000001

WORKLOADS = {
    # name: field, log_h, width, log_blowup, Poseidon2 width
    "babybear_2^22x256_b2": dict(field=0, log_h=22, width=256, log_blowup=1, p2w=16),
    "goldilocks_2^20x64_b4": dict(field=1, log_h=20, width=64, log_blowup=2, p2w=16),
    "goldilocks_2^20x64_b4_w12": dict(field=1, log_h=20, width=64, log_blowup=2, p2w=12),
    "babybear_2^14x16_b2": dict(field=0, log_h=14, width=16, log_blowup=1, p2w=16),
    # a smaller case of the default workload for profiler captures (inputs still > L2)
    "babybear_2^18x256_b2": dict(field=0, log_h=18, width=256, log_blowup=1, p2w=16),
    # the default workload's kernel instances (same NTT plan, same column chunks) on 16 columns,
    # for profiler captures (LDE 537 MB > L2)
    "babybear_2^22x16_b2": dict(field=0, log_h=22, width=16, log_blowup=1, p2w=16),
    # a smaller case of the Goldilocks workload for profiler captures (LDE 512 MB > L2)
    "goldilocks_2^18x64_b4": dict(field=1, log_h=18, width=64, log_blowup=2, p2w=16),
    # serving: Poisson arrivals of commit+FRI jobs, log2 rows uniform in [14, 24], widths in [32, 512]
    "serving_babybear": dict(kind="serving", field=0, log_h_lo=14, log_h_hi=24, w_lo=32, w_hi=512, log_blowup=1,
                             p2w=16, seed=5, jobs=60, slots=4, width=272, log_h=22),
    # batched form: 64 traces, log2 rows uniform in [12, 22], widths uniform in {8, ..., 256}
    "batch64_babybear": dict(kind="batch", field=0, n=64, log_h_lo=12, log_h_hi=22, w_step=8, w_hi=256,
                             log_blowup=1, p2w=16, seed=4, width=128, log_h=22),
    # many small traces (launch-bound as plain calls): 256 traces, log2 rows in [8, 14], widths {8..64}
    "batch256_small_babybear": dict(kind="batch", field=0, n=256, log_h_lo=8, log_h_hi=14, w_step=8, w_hi=64,
                                    log_blowup=1, p2w=16, seed=9, width=36, log_h=14),
    # the coset LDE alone under both tile-load modes of the NTT kernels (tensor copies, the
    # default, and coalesced loads into registers): (field, log_h, width, log_blowup)
    "lde_tile_loads": dict(kind="lde_sweep", field=0, log_h=22, width=256, log_blowup=1, p2w=16,
                           shapes=[(0, 22, 256, 1), (1, 20, 64, 2), (0, 20, 64, 1), (0, 18, 256, 1)]),
}
DEFAULT_WORKLOAD = "babybear_2^22x256_b2"
P2_SEED = 42
TRACE_SEED = 20240607
FRI = {"log_final": 8, "num_queries": 100, "challenge_seed": 7, "query_seed": 11}
ALPHA = [123456789, 987654321, 55555, 4242]
E2E_SLOTS = 4  # engine slots of the e2e leg: a job's H2D copy overlaps the other jobs' kernels
METRIC = "trace cells/s committed (LDE+Poseidon2 Merkle+FRI), batched vs plain; p99 ms"


def synthetic_trace(field: int, rows: int, width: int, seed: int, out=None):
    """Seeded uniform field elements as a row-major (rows, width) numpy array, the same on
    every machine: block k of 2^24 elements is numpy's exact bounded draw from
    default_rng([seed, k]), so blocks fill in parallel.  `out` (a numpy view of, e.g., a
    pinned buffer) receives the values in place."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    dt, p = (np.uint32, BB_P) if field == 0 else (np.uint64, GL_P)
    n = rows * width
    flat = np.empty(n, dt) if out is None else out.reshape(-1)
    assert flat.dtype == dt and flat.size == n
    block = 1 << 24

    def fill(k):
        off = k * block
        m = min(block, n - off)
        flat[off:off + m] = np.random.default_rng([seed, k]).integers(0, p, size=m, dtype=dt)

    with ThreadPoolExecutor(min(16, os.cpu_count() or 1)) as ex:
        list(ex.map(fill, range((n + block - 1) // block)))
    return flat.reshape(rows, width)


def p2_field_muls(field: int, p2w: int) -> int:
    """Algorithmic field multiplications of one permutation: 4 per S-box (x^7) on
    R_F*W + R_P lanes, W per internal round for the diagonal."""
    rf, rp = (8, 13) if field == 0 else (8, 22)
    return 4 * (rf * p2w + rp) + rp * p2w


def perms_of_commit(log_rows: int, width: int) -> tuple[int, int]:
    rows = 1 << log_rows
    return rows * ((width + 7) // 8), rows - 1  # leaf sponge perms, compressions


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ CPU legs
def cpu_commit_sample(wl: dict, log_rows: int, threads: int) -> tuple[float, int]:
    """Oracle (reference CPU path restated in C) commitment job — LDE + MMCS commit,
    and for BabyBear the alpha-reduction + FRI commit phase — of a 2^log_rows x width
    sample; returns (seconds, cells)."""
    import numpy as np

    import oracle as O

    O.build()
    O.set_threads(threads)
    rng = np.random.default_rng(TRACE_SEED)
    if wl["field"] == 0:
        t = rng.integers(0, BB_P, size=(1 << log_rows, wl["width"]), dtype=np.uint32)
    else:
        t = rng.integers(0, GL_P, size=(1 << log_rows, wl["width"]), dtype=np.uint64)
    h = O.hasher(wl["field"], P2_SEED, wl["p2w"])
    t0 = time.perf_counter()
    lde = O.coset_lde(wl["field"], t, wl["log_blowup"])
    O.mmcs_commit(h, [lde])
    if wl["field"] == 0 and wl.get("kind") != "batch":
        cw = O.combine_columns_ext4(lde, np.array(ALPHA, np.uint32))
        log_n = log_rows + wl["log_blowup"]
        O.fri_commit_ext4(cw, min(FRI["log_final"], log_n - 1), P2_SEED, FRI["challenge_seed"],
                          FRI["num_queries"], FRI["query_seed"])
    return time.perf_counter() - t0, t.size


def pick_cpu_sample(wl: dict, threads: int, budget_s: float) -> int:
    """Largest sample height whose commit fits the per-step budget (doubling)."""
    log_rows = 10
    dt, _ = cpu_commit_sample(wl, log_rows, threads)
    while log_rows < wl["log_h"] and dt * 2.2 < budget_s:
        log_rows += 1
        dt *= 2.1
    return log_rows


def run_reference(args, wl: dict, rank: int, world: int) -> int:
    """--impl reference: the reference's CPU path (oracle/ restatement) on host cores."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    log_rows = pick_cpu_sample(wl, threads, budget_s=4.0)
    for _ in range(args.warmup):
        cpu_commit_sample(wl, log_rows, threads)
    times = []
    cells = 0
    for _ in range(args.steps):
        dt, cells = cpu_commit_sample(wl, log_rows, threads)
        times.append(dt)
    total = sum(times)
    value = cells * len(times) / total
    fri_part = " + alpha-reduction + FRI commit phase and queries" if wl["field"] == 0 else ""
    sample = (f"2^{log_rows} x {wl['width']} trace per step (LDE x2^{wl['log_blowup']} + MMCS{fri_part}) of the "
              f"2^{wl['log_h']} x {wl['width']} {args.workload} job; value = cells of the sample / its time, "
              f"a rate measured on the smaller height, not extrapolated")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32" if wl["field"] == 0 else "u64", "data": "synthetic (seeded uniform field elements)",
        "config": {"workload": args.workload, "log_rows": wl["log_h"], "width": wl["width"],
                   "log_blowup": wl["log_blowup"], "poseidon2_width": wl["p2w"], "sample_log_rows": log_rows},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU path restated in C (oracle/, OpenMP over all host cores) with scalar u64/u128 "
                "remainder arithmetic per product, not p3's packed-SIMD Montgomery kernels, so it is slower "
                "than the reference's own CPU build would be; that build cannot be compiled here (no Rust "
                "toolchain, p3 0.4.2 crates absent)",
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------ ranks
class Ranks:
    """One process per GPU: the process group (NCCL on GPUs, gloo for the CPU tests),
    the barrier around timed regions and the max over ranks of a duration.  Replicas
    exchange nothing else: no data-path collective."""

    def __init__(self, world: int, device, backend: str = "nccl", timeout_s: int = 300):
        import torch

        self.torch = torch
        self.world = world
        self.device = device
        self.dist = None
        if world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()
        if self.device.type == "cuda":
            self.torch.cuda.synchronize()

    def max(self, x: float) -> float:
        if self.dist is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_rate(units_per_rank: float, steps: int, world: int, t_max: float) -> float:
    """Units all ranks processed / the slowest rank's time (weak scaling)."""
    return units_per_rank * steps * world / t_max


# ------------------------------------------------------------ GPU arm
def make_trace(torch, wl: dict, device):
    g = torch.Generator(device=device)
    g.manual_seed(TRACE_SEED)
    n, w = 1 << wl["log_h"], wl["width"]
    if wl["field"] == 0:
        return torch.randint(0, BB_P, (n, w), dtype=torch.int32, device=device, generator=g)
    hi = torch.randint(0, 1 << 32, (n, w), dtype=torch.int64, device=device, generator=g)
    lo = torch.randint(0, 1 << 32, (n, w), dtype=torch.int64, device=device, generator=g)
    v = (hi << 32) | lo  # uniform 64-bit pattern in int64 storage
    # reduce into [0, p): values >= p (as unsigned) are shifted down by p = 2^64 - 2^32 + 1
    eps = (1 << 32) - 1
    big = (v < 0) & (v >= -(1 << 32) + 1)
    return torch.where(big, v + eps, v)


def batch_shapes(wl: dict) -> list:
    import numpy as np

    rng = np.random.default_rng(wl["seed"])
    lh = rng.integers(wl["log_h_lo"], wl["log_h_hi"] + 1, size=wl["n"])
    ws = wl["w_step"] * rng.integers(1, wl["w_hi"] // wl["w_step"] + 1, size=wl["n"])
    return [(1 << int(a), int(b)) for a, b in zip(lh, ws)]


def fill_uniform(torch, field: int, shape, seed: int, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    if field == 0:
        return torch.randint(0, BB_P, shape, dtype=torch.int32, device=device, generator=g)
    return make_trace(torch, {"field": 1, "log_h": shape[0].bit_length() - 1, "width": shape[1]}, device)


def fill_pinned(torch, field: int, n: int, seed: int, device):
    """Pinned host buffer of n uniform field elements, generated on the device in 1 GB
    chunks (the device temporaries are released afterwards)."""
    dtype = torch.int32 if field == 0 else torch.int64
    out = torch.empty(n, dtype=dtype).pin_memory()
    chunk = (1 << 30) // out.element_size()
    for k, off in enumerate(range(0, n, chunk)):
        m = min(chunk, n - off)
        out[off:off + m].copy_(fill_uniform(torch, field, (m, 1), seed + k, device).view(-1).cpu())
    torch.cuda.empty_cache()
    return out


def golden_check(workload: str, wl: dict, root, pf) -> dict:
    """Compares the timed job's answers with the oracle's for the same seeded trace
    (tests/golden/fullsize.json, written by tests/golden/make_fullsize.py); a mismatch
    fails the run."""
    import hashlib

    import numpy as np

    key = "goldilocks_2^20x64_b4" if workload.startswith("goldilocks_2^20x64_b4") else workload
    try:
        with open(os.path.join(ROOT, "tests", "golden", "fullsize.json")) as f:
            g = json.load(f).get(key)
    except (OSError, ValueError):
        g = None
    if g is None:
        return {"checked": False, "why": "no oracle answers committed for this workload"}
    if wl["field"] == 1:
        want = g[f"root_w{wl['p2w']}"]
        assert [str(int(x)) for x in root] == want, "root differs from the oracle's"
        return {"checked": True, "compared": f"MMCS root (width-{wl['p2w']} Poseidon2) equal to the oracle's"}
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
    assert root.tolist() == g["root"], "root differs from the oracle's"
    assert pf.roots.tolist() == g["fri_roots"] and pf.betas.tolist() == g["fri_betas"], "FRI roots differ"
    assert pf.final.tolist() == g["fri_final"], "FRI final codeword differs"
    assert pf.query_indices.tolist() == g["query_indices"], "query indices differ"
    assert sha(pf.query_rows) == g["query_rows_sha256"], "query rows differ"
    assert sha(pf.query_siblings) == g["query_siblings_sha256"], "query paths differ"
    return {"checked": True, "compared": "trace root, every FRI root and beta, the final codeword and all "
                                         "query rows and paths of the last timed step equal to the oracle's"}


class GpuLocalMemory:
    """Within the block, the process runs on the host CPUs attached to the GPU's PCIe root
    (sysfs local_cpulist), so pinned pages first touched there sit in the GPU's NUMA node;
    the previous CPU set comes back afterwards."""

    def __init__(self, torch, device_index: int):
        self.cpus = None
        self.prev = None
        try:
            pr = torch.cuda.get_device_properties(device_index)
            bdf = "%04x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            with open(f"/sys/bus/pci/devices/{bdf}/local_cpulist") as f:
                cpus = set()
                for part in f.read().strip().split(","):
                    a, _, b = part.partition("-")
                    cpus.update(range(int(a), int(b or a) + 1))
            self.cpus = cpus & os.sched_getaffinity(0)
        except (OSError, ValueError, AttributeError):
            self.cpus = None

    def __enter__(self):
        if self.cpus:
            self.prev = os.sched_getaffinity(0)
            os.sched_setaffinity(0, self.cpus)
        return self

    def __exit__(self, *exc):
        if self.prev:
            os.sched_setaffinity(0, self.prev)

    def describe(self) -> str:
        return f"{len(self.cpus)} GPU-local host CPUs" if self.cpus else "GPU locality unknown (no sysfs entry)"


def measure_h2d(torch, pinned, dev, reps: int = 3) -> float:
    """Pinned host -> device copy bandwidth of the trace buffer on this box (GB/s, best of
    `reps`): 256 MiB pieces, one cudaMemcpyAsync each, as the engine uploads a job."""
    flat = pinned.view(-1)
    dst = torch.empty_like(flat, device=dev)
    piece = (256 << 20) // flat.element_size()
    s = torch.cuda.Stream(dev)
    best = 0.0
    with torch.cuda.stream(s):
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for off in range(0, flat.numel(), piece):
                dst[off:off + piece].copy_(flat[off:off + piece], non_blocking=True)
            e1.record(s)
            e1.synchronize()
            best = max(best, flat.numel() * flat.element_size() / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del dst
    return best


def load_traffic(workload: str):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(path)).get(workload)
    except (OSError, ValueError):
        return None


def run_ours(args, wl: dict, rank: int, world: int, local_rank: int) -> int:
    import ctypes as C

    import numpy as np
    import torch

    import ziros_b200 as Z
    from ziros_b200 import _native as N

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    N.check(N.load().zkb_set_device(local_rank))
    ranks = Ranks(world, dev, "nccl")
    dist = ranks.dist
    barrier, max_over_ranks = ranks.barrier, ranks.max

    field, lb = wl["field"], wl["log_blowup"]
    n, w = 1 << wl["log_h"], wl["width"]
    cells = n * w
    esize = 4 if field == 0 else 8
    pcs = Z.CudaTwoAdicPcs(field, P2_SEED, lb, wl["p2w"])
    # the seeded trace (the one tests/golden/fullsize.json answers for), in pinned host memory
    # first touched by the GPU's local CPUs
    local = GpuLocalMemory(torch, local_rank)
    with local:
        pinned = torch.empty((n, w), dtype=torch.int32 if field == 0 else torch.int64).pin_memory()
        synthetic_trace(field, n, w, TRACE_SEED, out=pinned.numpy().view(np.uint32 if field == 0 else np.uint64))
    trace = pinned.to(dev)
    torch.cuda.synchronize()
    h2d_gbs = measure_h2d(torch, pinned, dev)
    root = np.zeros(pcs.mmcs.digest_elems, dtype=np.uint32 if field == 0 else np.uint64)
    stream = torch.cuda.current_stream(dev)
    with_fri = field == 0

    def step_dev():
        if with_fri:
            _, _, pf = pcs.commit_fri_dev(trace, ALPHA, FRI["log_final"], FRI["num_queries"],
                                          FRI["challenge_seed"], FRI["query_seed"], want_tree=False, root=root)
            return pf
        pcs.commit_dev(trace, want_tree=False, root=root)
        return None

    engine = Z.CommitEngine(slots=E2E_SLOTS)
    fri_desc = dict(FRI, alpha=ALPHA) if with_fri else None

    def run_engine(k):
        ids = [engine.submit(pinned, field=field, seed=P2_SEED, log_blowup=lb, p2_width=wl["p2w"], fri=fri_desc,
                             host_ptr=pinned.data_ptr(), shape=(n, w)) for _ in range(k)]
        return [engine.wait(j) for j in ids]

    # ---- warm-up (builds twiddle/coset tables, fills the memory pool).  The engine's warm-up
    # runs at least two rounds of its slots, so that the memory pool and the block cache hold
    # what four jobs in flight use (growing the pool maps fresh device memory, which stalled
    # jobs for up to a second on some boxes); the device path's warm-up steps come after it,
    # directly before its timed region, so that they settle whatever blocks the engine's
    # jobs took over.
    fri_ref = step_dev()
    root_ref = root.copy()
    warm = run_engine(max(args.warmup, 2 * E2E_SLOTS))
    assert all((r[0] == root_ref).all() for r in warm), "engine root differs from the device path"
    for _ in range(max(args.warmup, 1)):
        fri_ref = step_dev()

    # ---- device-resident timed region (trace resident in HBM, > L2: no flush needed)
    sampler = ClockSampler(local_rank) if rank == 0 else None
    barrier()
    if sampler:
        sampler.start()
        time.sleep(0.4)
    N.profile_start()
    pool0 = N.pool_allocations()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    marks = []  # an event after every step: per-step device times (a stall shows as one long step)
    for _ in range(args.steps):
        last_pf = step_dev()
        marks.append(torch.cuda.Event(enable_timing=True))
        marks[-1].record(stream)
    ev1.record(stream)
    ev1.synchronize()
    barrier()
    kstats = N.profile_stop()
    clocks = sampler.stop() if sampler else None
    t_dev = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    pool_allocs = N.pool_allocations() - pool0
    step_ms = sorted(a.elapsed_time(b) for a, b in zip([ev0] + marks[:-1], marks))
    assert (root == root_ref).all(), "root changed between steps"
    assert not with_fri or (last_pf.roots == fri_ref.roots).all(), "FRI commitments changed between steps"
    gpu_launches = sum(v[0] for v in kstats.values())
    parity = golden_check(args.workload, wl, root, last_pf)

    # ---- end-to-end timed region: pinned host trace -> root and FRI answers on the host,
    # through the serving engine (the copy of one job overlaps the kernels of another)
    barrier()
    t0 = time.perf_counter()
    res = run_engine(args.steps)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    assert all((r[0] == root_ref).all() for r in res)
    e2e_lat = sorted(r[2]["latency_ms"] for r in res)
    engine.close()

    # ---- the workload's LDE with each tile-load mode of the NTT kernels (tensor copies,
    # the default, against coalesced loads into registers): best of 3 alternations of 5
    # LDEs each, outputs compared
    lde_out = torch.empty((n << lb, w), dtype=trace.dtype, device=dev)
    sp = C.c_void_p(stream.cuda_stream)
    shift = 31 if field == 0 else 7
    lde_ms, lde_ref = {}, None

    def lde():
        N.check(N.load().zkb_coset_lde_batch_dev(field, C.c_void_p(trace.data_ptr()), wl["log_h"], w, lb,
                                                 C.c_uint64(shift), 1, C.c_void_p(lde_out.data_ptr()), sp))

    for _ in range(3):
        for mode, key in ((0, "registers_ms"), (1, "tensor_copy_ms")):
            N.set_ntt_tile_loads(mode)
            lde()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(5):
                lde()
            e1.record(stream)
            e1.synchronize()
            lde_ms[key] = min(lde_ms.get(key, 1e30), e0.elapsed_time(e1) / 5)
            if lde_ref is None:
                lde_ref = lde_out.clone()
            else:
                assert torch.equal(lde_ref, lde_out), "tile-load modes give different LDEs"
    N.set_ntt_tile_loads(1)
    assert N.ntt_tile_load_errors() == 0
    del lde_out, lde_ref
    torch.cuda.empty_cache()

    # ---- integer-multiply ceiling for the Poseidon2 roofline (measured, this GPU)
    mul_peak = N.measure_mul_peak(field)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    value = whole_job_rate(cells, args.steps, world, t_dev)
    rounds = wl["log_h"] + lb - FRI["log_final"]
    fri_d2h = 4 * (8 * rounds + 4 * rounds + 4 * (1 << FRI["log_final"]) + FRI["num_queries"] * (
        2 + 8 * rounds + 8 * sum(wl["log_h"] + lb - r - 1 for r in range(rounds))))
    e2e = cells * args.steps * world / t_e2e
    ceiling_ms = max(1e3 * t_dev / args.steps, cells * esize / (h2d_gbs * 1e9) * 1e3)
    # roofline of the dominant kernel (leaf sponge hashing; integer-multiply bound)
    N_rows = n << lb
    leaf_perms, comp_perms = perms_of_commit(wl["log_h"] + lb, w)
    lk = kstats.get("merkle_leaf_hash", (1, float("nan"), 0))
    leaf_ms = lk[1] / max(lk[0], 1)
    muls = leaf_perms * p2_field_muls(field, wl["p2w"])
    achieved = muls / (leaf_ms * 1e-3) / 1e9
    traffic = load_traffic(args.workload)
    roofline = {
        "kernel": "merkle_leaf_hash", "bound": "int", "unit": "Gmul/s",
        "achieved": achieved, "peak": mul_peak / 1e9, "frac": achieved / (mul_peak / 1e9),
        "peak_source": "measured in this run: zkb_measure_mul_peak (independent field-multiply chains on all SMs)",
        "work_per_launch": f"{leaf_perms} Poseidon2 perms x {p2_field_muls(field, wl['p2w'])} field mults",
        "traffic": traffic.get("merkle_leaf_hash") if traffic else None,
    }
    # HBM roofline of the NTT passes (each pass reads and writes its tiles once)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm_peak, hbm_src = float(peaks["hbm_gbs"]), "of measured"
    except (OSError, ValueError, KeyError):
        hbm_peak, hbm_src = 6650.0, "of fallback"
    # NTT kernels: plain passes read and write their tiles once; the fused kernel reads the
    # coefficient matrix once and writes every coset block once
    kmax = 10 if field == 0 else 7  # largest pass of the library's default plans
    n_pass = -(-wl["log_h"] // kmax)
    b_blocks = 1 << lb
    ntt_roof = []

    def kstat(*names):
        """(launches, total ms, max ms) summed over the kernels of these names (register or
        tensor-copy tile loads)."""
        got = [kstats[k] for k in names if k in kstats]
        if not got:
            return None
        return (sum(g[0] for g in got), sum(g[1] for g in got), max(g[2] for g in got))

    tile_loads = "tensor copy" if ("ntt_pass_tma" in kstats or "lde_fused_tma" in kstats) else "registers"
    nk = kstat("ntt_pass", "ntt_pass_tma")
    if nk and n_pass > 1:
        bytes_per_step = 2 * esize * (n * w * (n_pass - 1) + N_rows * w * (n_pass - 1))
        per_launch = bytes_per_step * args.steps / nk[0]
        ach = per_launch / (nk[1] / nk[0] * 1e-3) / 1e9
        ntt_roof.append({"kernel": "ntt_pass", "tile_loads": tile_loads, "bound": "hbm", "unit": "GB/s",
                         "achieved": ach, "peak": hbm_peak,
                         "frac": ach / hbm_peak, "peak_source": hbm_src,
                         "algorithmic_bytes_per_launch": per_launch,
                         "traffic": traffic.get("ntt_pass") if traffic else None})
    fk = kstat("lde_fused", "lde_fused_tma")
    if fk:
        per_launch = esize * (n * w + b_blocks * n * w)
        ach = per_launch / (fk[1] / fk[0] * 1e-3) / 1e9
        ntt_roof.append({"kernel": "lde_fused", "tile_loads": tile_loads, "bound": "hbm", "unit": "GB/s",
                         "achieved": ach, "peak": hbm_peak,
                         "frac": ach / hbm_peak, "peak_source": hbm_src,
                         "algorithmic_bytes_per_launch": per_launch,
                         "traffic": traffic.get("lde_fused") if traffic else None})

    # ---- CPU baseline (oracle on host cores, bounded sample)
    cpu = None
    if world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        log_rows = pick_cpu_sample(wl, threads, budget_s=8.0)
        dts = []
        for _ in range(2):
            dt, c = cpu_commit_sample(wl, log_rows, threads)
            dts.append(dt)
        job = f"LDE x2^{lb} + MMCS" + (" + alpha-reduction + FRI commit phase and queries" if with_fri else "")
        cpu = {"value": c / min(dts), "unit": "cells/s", "cores": threads, "kind": "port",
               "sample": f"2^{log_rows} x {w} trace ({job}), best of 2, oracle/ C restatement with scalar "
                         "remainder arithmetic (not p3's packed-SIMD kernels)"}

    line = {
        "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32" if field == 0 else "u64",
        "data": "synthetic (seeded uniform field elements)",
        "config": {"workload": args.workload, "log_rows": wl["log_h"], "width": wl["width"],
                   "log_blowup": wl["log_blowup"], "poseidon2_width": wl["p2w"],
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (trace %.1f GB, LDE %.1f GB)" % (cells * esize / 1e9,
                                                                             N_rows * w * esize / 1e9)},
        "e2e": {"value": e2e, "unit": "cells/s", "h2d_bytes_per_step": cells * esize,
                "d2h_bytes_per_step": int(root.nbytes) + (fri_d2h if with_fri else 0),
                "ms_per_step": 1e3 * t_e2e / args.steps, "path": f"zkb_engine_submit/wait, {E2E_SLOTS} slots",
                "warmup_jobs": max(args.warmup, 2 * E2E_SLOTS),
                "latency_ms_p50": e2e_lat[len(e2e_lat) // 2], "latency_ms_max": e2e_lat[-1],
                "h2d_gbs_measured": h2d_gbs, "pinned_memory": local.describe(),
                "ceiling_ms": ceiling_ms, "frac_of_ceiling": ceiling_ms / (1e3 * t_e2e / args.steps),
                "ceiling": "max(device ms/step, trace bytes / measured pinned H2D bandwidth): the copy of "
                           "one job hidden under another's kernels"},
        "parity": parity,
        "roofline": roofline,
        "roofline_ntt": ntt_roof,
        "lde_tile_loads": dict({k: round(v, 3) for k, v in lde_ms.items()},
                               what="the workload's coset LDE alone (zkb_coset_lde_batch_dev), best of 3 x 5"),
        "step": "LDE + Poseidon2 MMCS" + (" + alpha-reduction + FRI (2^%d -> 2^%d, %d queries)" % (
            wl["log_h"] + lb, FRI["log_final"], FRI["num_queries"]) if with_fri else ""),
        "cpu_baseline": cpu,
        "gpu_launches": gpu_launches,
        "kernels": {k: {"launches": v[0], "ms_total": round(v[1], 3), "ms_max": round(v[2], 3)}
                    for k, v in sorted(kstats.items(), key=lambda kv: -kv[1][1])},
        # per-step device time (min / median / max) and the part of a step no kernel of the
        # library covered (host turnaround between launches and between steps)
        "step_ms": {"min": round(step_ms[0], 3), "median": round(step_ms[len(step_ms) // 2], 3),
                    "max": round(step_ms[-1], 3),
                    "idle_per_step": round(1e3 * t_dev / args.steps - sum(v[1] for v in kstats.values()) / args.steps,
                                           3),
                    "pool_allocations": pool_allocs},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_batch(args, wl: dict, rank: int, world: int, local_rank: int) -> int:
    """Batched form: 64 uneven BabyBear traces committed by one plan (one CUDA graph per
    step, autotuned kernel shapes) against the plain path (64 zkb_pcs_commit_dev calls)
    on the same GPU and the same device-resident traces."""
    import ctypes as C

    import numpy as np
    import torch

    import ziros_b200 as Z
    from ziros_b200 import _native as N

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = N.load()
    N.check(lib.zkb_set_device(local_rank))
    ranks = Ranks(world, dev, "nccl")
    dist = ranks.dist
    barrier, max_over_ranks = ranks.barrier, ranks.max

    field, lb, p2w = wl["field"], wl["log_blowup"], wl["p2w"]
    shapes = batch_shapes(wl)
    cells = sum(h * w for h, w in shapes)
    esize = 4 if field == 0 else 8
    stream = torch.cuda.current_stream(dev)
    sp = C.c_void_p(stream.cuda_stream)
    t0 = time.perf_counter()
    batch = Z.BatchCommit(shapes, field=field, seed=P2_SEED, log_blowup=lb, p2_width=p2w, use_graph=True,
                          autotune=True)
    create_s = time.perf_counter() - t0
    info = batch.info()
    # traces generated on the device straight into the plan's input buffers
    ptrs = []
    for i, (h, w) in enumerate(shapes):
        t = fill_uniform(torch, field, (h, w), TRACE_SEED + i, dev)
        batch.copy_in(i, t)
        p = C.c_void_p()
        N.check(lib.zkb_batch_trace_ptr(batch._h, i, C.byref(p)))
        ptrs.append(p)
        del t
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    hasher = N.Hasher(field, p2w, P2_SEED)
    digest = 8 if p2w == 16 else 4
    dt = np.uint32 if field == 0 else np.uint64
    plain_roots = np.zeros((len(shapes), digest), dtype=dt)

    def plain_step():
        for i, (h, w) in enumerate(shapes):
            N.check(lib.zkb_pcs_commit_dev(C.byref(hasher), ptrs[i], h.bit_length() - 1, w, lb,
                                           plain_roots[i].ctypes.data_as(C.c_void_p), None, sp))

    def batch_step():
        batch.run(sp)

    def timed(fn, k):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / 1e3)

    for _ in range(max(args.warmup, 1)):
        plain_step()
        batch_step()
    got = batch.roots(sp)
    assert (got == plain_roots).all(), "batched roots differ from the plain per-trace commits"

    N.profile_start()
    t_plain = timed(plain_step, args.steps)
    kstats = N.profile_stop()
    plain_launches = sum(v[0] for v in kstats.values())
    sampler = ClockSampler(local_rank) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.4)
    t_batch = timed(batch_step, args.steps)
    clocks = sampler.stop() if sampler else None
    assert (batch.roots(sp) == plain_roots).all()

    # end to end: traces from pinned host memory (one pinned buffer of the largest trace
    # serves every trace), H2D copies + run + root read-back inside the timed region;
    # zkb_batch_run_host overlaps the copies with the commitment, the serial form copies
    # every trace first and then replays the graph
    hmax = max(h * w for h, w in shapes)
    pinned = fill_pinned(torch, field, hmax, TRACE_SEED, dev)
    srcs = (C.c_void_p * len(shapes))(*([pinned.data_ptr()] * len(shapes)))

    def e2e_step():
        N.check(lib.zkb_batch_run_host(batch._h, srcs, sp))
        return batch.roots(sp)

    def e2e_serial_step():
        for i in range(len(shapes)):
            N.check(lib.zkb_batch_copy_in(batch._h, i, srcs[i], 0, sp))
        batch.run(sp)
        return batch.roots(sp)

    def wall(fn):
        fn()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r = fn()
        return max_over_ranks(time.perf_counter() - t0), r

    t_e2e, r_host = wall(e2e_step)
    t_e2e_serial, r_serial = wall(e2e_serial_step)
    assert (r_host == r_serial).all(), "run_host roots differ from copy-in + graph run on the same sources"
    batch.close()  # the persistent plan below needs the memory
    del batch

    # ---- the persistent form: ONE kernel per run fed by a device work queue (autotuned
    # Merkle-level fusion), on traces generated straight into its input buffers
    pers = None
    if field == 0 and p2w == 16 and all(w % 8 == 0 for _, w in shapes):
        N.release_cached_memory()
        t0 = time.perf_counter()
        pb = Z.BatchCommit(shapes, field=field, seed=P2_SEED, log_blowup=lb, p2_width=p2w, persistent=True,
                           autotune=True)
        pcreate_s = time.perf_counter() - t0
        for i, (h, w) in enumerate(shapes):
            t = fill_uniform(torch, field, (h, w), TRACE_SEED + i, dev)
            pb.copy_in(i, t)
            del t
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        for _ in range(max(args.warmup, 1)):
            pb.run(sp)
        assert (pb.roots(sp) == plain_roots).all(), "persistent-form roots differ from the plain commits"
        t_pers = timed(lambda: pb.run(sp), args.steps)
        assert (pb.roots(sp) == plain_roots).all()
        prof = pb.profile(sp)
        q = pb.queue_info()
        pers = {"value": cells * args.steps * world / t_pers, "ms_per_step": 1e3 * t_pers / args.steps,
                "vs_graph": t_batch / t_pers, "vs_plain": t_plain / t_pers, "work_queue": q,
                "plan_create_s": pcreate_s, "tune_ms": pb.info()["tune_ms"],
                "profile_block_ms": {k: round(v / (q["grid"] if k != "span_ms" else 1), 2) for k, v in prof.items()},
                "path": "one persistent kernel per run (device work queue of NTT / leaf-hash / compression tiles, "
                        "bounded waits on per-step counters) captured in a CUDA graph"}
        pb.close()
        del pb
        N.release_cached_memory()
    # the plain path end to end: one host-pointer commit per trace
    pcs = Z.CudaTwoAdicPcs(field, P2_SEED, lb, p2w)
    r = np.zeros(digest, dtype=dt)
    pcs.commit_ptr(pinned.data_ptr(), shapes[0][0], shapes[0][1], want_tree=False, root=r)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for h, w in shapes:
            pcs.commit_ptr(pinned.data_ptr(), h, w, want_tree=False, root=r)
    t_e2e_plain = max_over_ranks(time.perf_counter() - t0)

    mul_peak = N.measure_mul_peak(field)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    muls = 0
    for h, w in shapes:
        lp, cp = perms_of_commit((h << lb).bit_length() - 1, w)
        muls += (lp + cp) * p2_field_muls(field, p2w)
    value = whole_job_rate(cells, args.steps, world, t_batch)
    plain = cells * args.steps * world / t_plain
    ach = muls * args.steps / t_batch / 1e9
    cpu = None
    if world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        cwl = dict(kind="batch", field=field, width=128, log_blowup=lb, p2w=p2w, log_h=22)
        log_rows = pick_cpu_sample(cwl, threads, budget_s=8.0)
        dts = [cpu_commit_sample(dict(cwl, field=field), log_rows, threads) for _ in range(2)]
        best = min(dts)
        cpu = {"value": best[1] / best[0], "unit": "cells/s", "cores": threads, "kind": "port",
               "sample": f"2^{log_rows} x 128 trace (the batch's mean width; LDE x2^{lb} + MMCS), best of 2, "
                         "oracle/ C restatement"}
    line = {
        "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_batch / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32" if field == 0 else "u64",
        "data": "synthetic (seeded uniform field elements)",
        "config": {"workload": args.workload, "n_traces": len(shapes), "log_rows": [wl["log_h_lo"], wl["log_h_hi"]],
                   "widths": [wl["w_step"], wl["w_hi"]], "shape_seed": wl["seed"], "total_cells": cells,
                   "log_blowup": lb, "poseidon2_width": p2w, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (%.1f GB of traces)" % (cells * esize / 1e9),
                   "branches": info["branches"], "leaf_threads": info["leaf_threads"],
                   "graph_kernels": info["kernels_per_run"], "plan_device_gb": info["device_bytes"] / 1e9,
                   "plan_create_s": create_s, "tune_ms": info["tune_ms"]},
        "plain": {"value": plain, "ms_per_step": 1e3 * t_plain / args.steps,
                  "launches_per_step": plain_launches / args.steps,
                  "path": f"{len(shapes)} x zkb_pcs_commit_dev on the same device-resident traces"},
        "batched_vs_plain": value / plain,
        "persistent": pers,
        "e2e": {"value": cells * args.steps * world / t_e2e, "unit": "cells/s",
                "h2d_bytes_per_step": cells * esize, "d2h_bytes_per_step": len(shapes) * digest * esize,
                "ms_per_step": 1e3 * t_e2e / args.steps,
                "path": "zkb_batch_run_host (pinned sources; copies overlapped with the LDEs and per-trace "
                        "trees) + zkb_batch_roots",
                "serial_ms_per_step": 1e3 * t_e2e_serial / args.steps,
                "serial_path": f"zkb_batch_copy_in (pinned) x{len(shapes)} + zkb_batch_run + zkb_batch_roots",
                "device_ms_per_step": 1e3 * t_batch / args.steps,
                "plain_value": cells * args.steps * world / t_e2e_plain,
                "plain_path": f"{len(shapes)} x zkb_pcs_commit from pinned host memory"},
        "roofline": {"kernel": "whole batched step (LDE + leaf hashing + compression)", "bound": "int",
                     "unit": "Gmul/s", "achieved": ach, "peak": mul_peak / 1e9, "frac": ach / (mul_peak / 1e9),
                     "peak_source": "measured in this run: zkb_measure_mul_peak",
                     "work_per_step": f"{muls} Poseidon2 field mults", "traffic": None},
        "cpu_baseline": cpu,
        "gpu_launches": info["kernels_per_run"] * args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def run_sharded(args, wl: dict, rank: int, world: int, local_rank: int) -> int:
    """One commitment of the workload's trace split over the ranks (ziros_b200.sharded):
    each rank extends its columns, one all-to-all moves row blocks, each rank hashes its
    rows, the subtree roots are gathered; with FRI the reduced codeword is gathered and
    folded on every rank.  The trace is fixed as ranks are added (strong scaling)."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    from ziros_b200 import _native as N
    from ziros_b200 import sharded as S

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    N.check(N.load().zkb_set_device(local_rank))
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    field, lb = wl["field"], wl["log_blowup"]
    n, w = 1 << wl["log_h"], wl["width"]
    c0, c1 = S.column_ranges(w, world)[rank]
    cols = fill_uniform(torch, field, (n, c1 - c0), TRACE_SEED + rank, dev)
    ops = S.CudaShardOps(field, P2_SEED, lb, wl["p2w"], dev)
    fri = S.FriArgs(FRI["log_final"], FRI["num_queries"], ALPHA, FRI["challenge_seed"], FRI["query_seed"]) \
        if field == 0 else None
    stream = torch.cuda.current_stream(dev)
    for _ in range(max(args.warmup, 1)):
        ref = S.commit_sharded(cols, w, ops, fri=fri).root
    sampler = ClockSampler(local_rank) if rank == 0 else None
    barrier()
    if sampler:
        sampler.start()
        time.sleep(0.4)
    N.profile_start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        res = S.commit_sharded(cols, w, ops, fri=fri)
    ev1.record(stream)
    ev1.synchronize()
    barrier()
    kstats = N.profile_stop()
    clocks = sampler.stop() if sampler else None
    t = ev0.elapsed_time(ev1) / 1e3
    if world > 1:
        tt = torch.tensor([t], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    assert np.array_equal(res.root, ref), "root changed between steps"
    del res
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    esize = 4 if field == 0 else 8
    line = {
        "metric": METRIC, "value": n * w * args.steps / t, "unit": "cells/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32" if field == 0 else "u64",
        "data": "synthetic (seeded uniform field elements; each rank generates its own columns)",
        "config": {"workload": args.workload, "log_rows": wl["log_h"], "width": w, "log_blowup": lb,
                   "poseidon2_width": wl["p2w"],
                   "parallelism": f"one commitment over {world} ranks: column-sharded LDE, all-to-all of "
                                  f"row blocks, row-sharded hashing",
                   "l2": "inputs larger than L2 (trace %.1f GB)" % (n * w * esize / 1e9)},
        "e2e": None,
        "note": "device-resident only: the trace starts in each rank's HBM",
        "gpu_launches": sum(v[0] for v in kstats.values()),
        "kernels": {k: {"launches": v[0], "ms_total": round(v[1], 3)}
                    for k, v in sorted(kstats.items(), key=lambda kv: -kv[1][1])},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def serving_jobs(wl: dict, n: int, seed: int) -> list:
    import numpy as np

    rng = np.random.default_rng(seed)
    lh = rng.integers(wl["log_h_lo"], wl["log_h_hi"] + 1, size=n)
    ws = rng.integers(wl["w_lo"], wl["w_hi"] + 1, size=n)
    return [(1 << int(a), int(b)) for a, b in zip(lh, ws)]


def run_serving(args, wl: dict, rank: int, world: int, local_rank: int) -> int:
    """Serving form: a Poisson stream of BabyBear commit+FRI jobs of mixed sizes through
    the continuous-batching engine (admission by free HBM, `slots` jobs in flight, state
    device-resident through FRI) at swept arrival rates, against the plain path: the same
    stream through a one-slot engine (one job at a time, FIFO).  Every job's root and FRI
    commitments must be the same in both."""
    import threading as th

    import numpy as np
    import torch

    import ziros_b200 as Z
    from ziros_b200 import _native as N

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    N.check(N.load().zkb_set_device(local_rank))
    if world > 1 and rank != 0:
        return 0  # serving replicas are independent; rank 0 reports its own
    field, lb = wl["field"], wl["log_blowup"]
    fri = dict(FRI, alpha=ALPHA)
    hmax = (1 << wl["log_h_hi"]) * wl["w_hi"]
    pinned = fill_pinned(torch, field, hmax, TRACE_SEED, dev)
    torch.cuda.synchronize()

    def drive(engine, jobs, rate, seed):
        """Submits the jobs at Poisson arrival times (rate 0: all at once)."""
        rng = np.random.default_rng(seed)
        gaps = rng.exponential(1.0 / rate, size=len(jobs)) if rate > 0 else np.zeros(len(jobs))
        ids = [None] * len(jobs)
        failed = []
        t_start = time.perf_counter()

        def submitter():
            t = t_start
            try:
                for i, (h, w) in enumerate(jobs):
                    t += gaps[i]
                    d = t - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    ids[i] = engine.submit(pinned, host_ptr=pinned.data_ptr(), shape=(h, w), fri=fri)
            except Exception as e:  # surfaced by the waiting loop below
                failed.append(e)

        sub = th.Thread(target=submitter)
        sub.start()
        res = []
        for i in range(len(jobs)):
            while ids[i] is None:
                if failed:
                    sub.join()
                    raise failed[0]
                time.sleep(0.0005)
            res.append(engine.wait(ids[i]))
        sub.join()
        return res, time.perf_counter() - t_start

    def summarize(jobs, res, span):
        lat = np.array([r[2]["latency_ms"] for r in res])
        cells = sum(h * w for h, w in jobs)
        return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "cells_per_s": cells / span, "span_s": span, "jobs": len(jobs)}

    # service time of the plain path: the calibration list back to back on one slot
    calib = serving_jobs(wl, wl["jobs"], wl["seed"])
    eng1 = Z.CommitEngine(slots=1, policy="fifo")
    engN = Z.CommitEngine(slots=wl["slots"])  # the engine's default admission: oldest fitting job first
    engS = Z.CommitEngine(slots=wl["slots"], policy="smallest")
    drive(eng1, calib[:4], 0, 1)  # warm-up: tables, memory pool
    _, span = drive(eng1, calib, 0, 2)
    service_s = span / len(calib)
    mu = 1.0 / service_s
    rates = [0.5 * mu, 0.8 * mu, 1.0 * mu, 1.5 * mu]
    drive(engN, calib[:4], 0, 3)
    drive(engS, calib[:4], 0, 4)
    sweep = []
    h2d = 0
    sampler = ClockSampler(local_rank)
    sampler.start()
    for k, rate in enumerate(rates):
        jobs = serving_jobs(wl, wl["jobs"], wl["seed"] + 100 + k)
        r_b, s_b = drive(engN, jobs, rate, 1000 + k)
        r_s, s_s = drive(engS, jobs, rate, 1000 + k)
        r_p, s_p = drive(eng1, jobs, rate, 1000 + k)
        for a, b, c in zip(r_b, r_p, r_s):
            assert (a[0] == b[0]).all() and (a[1].roots == b[1].roots).all(), "a result differs in the mix"
            assert (c[0] == b[0]).all() and (c[1].roots == b[1].roots).all(), "a result differs in the mix"
        sweep.append({"rate_jobs_per_s": rate, "load": rate / mu, "batched": summarize(jobs, r_b, s_b),
                      "batched_smallest": summarize(jobs, r_s, s_s), "plain": summarize(jobs, r_p, s_p)})
        h2d = 4 * sum(h * w for h, w in jobs)
    clocks = sampler.stop()
    st = engN.stats()
    eng1.close()
    engN.close()
    engS.close()
    top = sweep[-1]
    line = {
        "metric": METRIC, "value": top["batched"]["cells_per_s"], "unit": "cells/s", "n_gpus": 1,
        "steps": len(rates), "warmup": 4, "ms_per_step": 1e3 * top["batched"]["span_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded uniform field elements; Poisson arrivals)",
        "config": {"workload": args.workload, "log_rows": [wl["log_h_lo"], wl["log_h_hi"]],
                   "widths": [wl["w_lo"], wl["w_hi"]], "jobs_per_rate": wl["jobs"], "slots": wl["slots"],
                   "log_blowup": lb, "fri": {"log_final": FRI["log_final"], "queries": FRI["num_queries"]},
                   "hbm_budget_gb": st["hbm_budget"] / 1e9, "hbm_peak_gb": st["hbm_peak"] / 1e9,
                   "pinned_host_gb": hmax * 4 / 1e9, "service_ms_plain": 1e3 * service_s,
                   "l2": "inputs larger than L2"},
        "p50_ms": top["batched"]["p50_ms"], "p99_ms": top["batched"]["p99_ms"],
        "policies": {"batched": f"{wl['slots']} slots, oldest fitting job first (the engine default), a job "
                                f"passed over {N.ADMIT_MAX_BYPASS} times goes next",
                     "batched_smallest": f"{wl['slots']} slots, fewest cells first, same bypass bound",
                     "plain": "1 slot, FIFO"},
        "batched_smallest": top["batched_smallest"],
        "plain": top["plain"],
        "sweep": sweep,
        "e2e": {"value": top["batched"]["cells_per_s"], "unit": "cells/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": None,
                "path": "zkb_engine_submit/wait from pinned host memory (every number here is end to end)"},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_lde_sweep(args, wl: dict, rank: int, world: int, local_rank: int) -> int:
    """The coset LDE (zkb_coset_lde_batch_dev, rows bit-reversed) of each shape under both
    tile-load modes of the NTT kernels, alternating the modes: best of `steps` rounds of 10
    LDEs each after `warmup` untimed ones; the outputs of the two modes are compared."""
    import ctypes as C

    import numpy as np
    import torch

    from ziros_b200 import _native as N

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    lib = N.load()
    N.check(lib.zkb_set_device(local_rank))
    stream = torch.cuda.current_stream(dev)
    sp = C.c_void_p(stream.cuda_stream)
    out_rows = []
    for field, log_h, w, lb in wl["shapes"]:
        n = 1 << log_h
        t = fill_uniform(torch, field, (n, w), TRACE_SEED, dev)
        out = torch.empty((n << lb, w), dtype=t.dtype, device=dev)
        shift = 31 if field == 0 else 7

        def lde():
            N.check(lib.zkb_coset_lde_batch_dev(field, C.c_void_p(t.data_ptr()), log_h, w, lb, C.c_uint64(shift), 1,
                                                C.c_void_p(out.data_ptr()), sp))

        best, ref = {}, None
        for _ in range(max(args.steps, 1)):
            for mode, key in ((0, "registers_ms"), (1, "tensor_copy_ms")):
                N.set_ntt_tile_loads(mode)
                for _ in range(max(args.warmup, 1)):
                    lde()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(10):
                    lde()
                e1.record(stream)
                e1.synchronize()
                best[key] = min(best.get(key, 1e30), e0.elapsed_time(e1) / 10)
                if ref is None:
                    ref = out.clone()
                else:
                    assert torch.equal(ref, out), "tile-load modes give different LDEs"
        N.set_ntt_tile_loads(1)
        out_rows.append(dict(field="babybear" if field == 0 else "goldilocks", log_h=log_h, width=w, log_blowup=lb,
                             registers_ms=round(best["registers_ms"], 4),
                             tensor_copy_ms=round(best["tensor_copy_ms"], 4),
                             speedup=round(best["registers_ms"] / best["tensor_copy_ms"], 4)))
        del t, out, ref
        torch.cuda.empty_cache()
    assert N.ntt_tile_load_errors() == 0
    if rank == 0:
        speed = [r["speedup"] for r in out_rows]
        gm = float(np.exp(np.mean(np.log(speed))))
        print(json.dumps({"metric": "coset LDE time, tensor-copy vs register tile loads (geometric-mean speed-up)",
                          "value": gm, "unit": "x", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                          "higher_is_better": True, "vs_baseline": None, "data": "synthetic (seeded uniform)",
                          "config": {"workload": args.workload}, "shapes": out_rows}), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--skip-cpu", action="store_true", help="omit the cpu_baseline leg")
    ap.add_argument("--sharded", action="store_true",
                    help="one commitment split over the ranks (strong scaling) instead of replicas")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, wl, rank, world)
    if wl.get("kind") == "batch":
        return run_batch(args, wl, rank, world, local_rank)
    if wl.get("kind") == "serving":
        return run_serving(args, wl, rank, world, local_rank)
    if wl.get("kind") == "lde_sweep":
        return run_lde_sweep(args, wl, rank, world, local_rank)
    if args.sharded:
        return run_sharded(args, wl, rank, world, local_rank)
    return run_ours(args, wl, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
