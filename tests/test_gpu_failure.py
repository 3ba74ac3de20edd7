"""Failure detection: the watchdog, the circuit breaker and job cancellation.

Faults are made on the host only (zkb_debug_inject_fault): an allocation that reports
out-of-memory, a stream wait that reports an expired deadline after the work has
finished.  No test faults, traps or hangs the GPU.  The circuit is process-wide, so
every test closes it again before it ends."""
import numpy as np
import pytest

import ziros_b200 as Z
from ziros_b200 import _native as N
from conftest import rand_field

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def closed_circuit():
    N.circuit_reset()
    N.inject_fault(1, 0)
    N.inject_fault(2, 0)
    yield
    N.inject_fault(1, 0)
    N.inject_fault(2, 0)
    N.circuit_reset()


def _commit(trace):
    return Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1).commit(trace)[0]


def test_out_of_memory_is_an_error_not_a_device_fault(oracle):
    trace = rand_field(Z.BABYBEAR, (1 << 9, 8), 1)
    N.inject_fault(1, 1)
    with pytest.raises(Z.ZkbError) as e:
        _commit(trace)
    assert e.value.code == N.ERR_OOM and "out of memory" in str(e.value)
    assert N.circuit_open()[0] is False  # the device is fine: later calls proceed
    lde = oracle.coset_lde(Z.BABYBEAR, trace, 1)
    assert (_commit(trace) == oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [lde])[-1][0]).all()


def test_watchdog_opens_the_circuit_and_calls_decline_until_reset(oracle):
    trace = rand_field(Z.BABYBEAR, (1 << 9, 8), 2)
    N.inject_fault(2, 1)
    with pytest.raises(Z.ZkbError) as e:
        _commit(trace)
    assert e.value.code == N.ERR_TIMEOUT
    is_open, why = N.circuit_open()
    assert is_open and "watchdog" in why
    # the reference's fallback signal: declined, the caller takes its CPU path
    with pytest.raises(Z.ZkbDeclined) as d:
        _commit(trace)
    assert "circuit open" in str(d.value)
    states = np.zeros(16, np.uint32)
    rc, ne, ni = Z.round_constants(Z.BABYBEAR, 42)
    assert Z.CudaPoseidon2().batch_permute_babybear(states, rc, ne, ni) is False
    with pytest.raises(Z.ZkbDeclined):
        Z.BatchCommit([(1 << 4, 8)], autotune=False)
    N.circuit_reset()
    lde = oracle.coset_lde(Z.BABYBEAR, trace, 1)
    assert (_commit(trace) == oracle.mmcs_commit(oracle.hasher(Z.BABYBEAR, 42), [lde])[-1][0]).all()


def test_engine_job_reports_the_timeout_and_the_engine_declines_new_jobs():
    eng = Z.CommitEngine(slots=1)
    try:
        N.inject_fault(2, 1)
        jid = eng.submit(rand_field(Z.BABYBEAR, (1 << 10, 16), 3))
        with pytest.raises(Z.ZkbError) as e:
            eng.wait(jid)
        assert e.value.code == N.ERR_TIMEOUT
        with pytest.raises(Z.ZkbDeclined):
            eng.submit(rand_field(Z.BABYBEAR, (1 << 10, 16), 4))
        N.circuit_reset()
        root, _, _ = eng.wait(eng.submit(rand_field(Z.BABYBEAR, (1 << 10, 16), 4)))
        assert root.shape == (8,)
    finally:
        eng.close()


def test_cancel_a_queued_job():
    """A budget that fits one job at a time keeps the later jobs queued; cancelling one
    of them ends its wait with ERR_CANCELLED and the others complete."""
    n, w = 1 << 18, 64  # ~10 ms of device work per job: the queue outlives the submits
    # the engine's estimate: staged trace + LDE + digest layers + 64 MiB
    per_job = n * w * 4 + 2 * n * w * 4 + 2 * (2 * n) * 64 + (64 << 20)
    eng = Z.CommitEngine(slots=1, hbm_budget=int(per_job * 1.5))
    try:
        traces = [rand_field(Z.BABYBEAR, (n, w), 10 + k) for k in range(4)]
        ids = [eng.submit(t) for t in traces]
        assert eng.cancel(ids[3]) is True
        with pytest.raises(Z.ZkbError) as e:
            eng.wait(ids[3])
        assert e.value.code == N.ERR_CANCELLED
        roots = [eng.wait(j)[0] for j in ids[:3]]
        want = [Z.CudaTwoAdicPcs(Z.BABYBEAR, 42, 1).commit(t)[0] for t in traces[:3]]
        assert all((a == b).all() for a, b in zip(roots, want))
        with pytest.raises(Z.ZkbError):  # a finished job is no longer known to the engine
            eng.cancel(ids[0])
    finally:
        eng.close()


def test_thresholds_decline_small_host_calls(oracle):
    """Below a threshold a host-pointer call declines (the caller's CPU path runs); at or
    above it the call runs on the device as before."""
    rc, ne, ni = Z.round_constants(Z.BABYBEAR, 42)
    p2 = Z.CudaPoseidon2()
    dft = Z.CudaDft(Z.BABYBEAR)
    try:
        N.set_thresholds(ntt=1 << 10, poseidon2=1000)
        assert p2.batch_permute_babybear(np.zeros(16 * 10, np.uint32), rc, ne, ni) is False
        big = rand_field(Z.BABYBEAR, 16 * 1000, 7)
        want = oracle.permute(Z.BABYBEAR, big, rc, ne, ni)
        assert p2.batch_permute_babybear(big, rc, ne, ni) is True and (big == want).all()
        with pytest.raises(Z.ZkbDeclined) as e:
            dft.dft_batch(rand_field(Z.BABYBEAR, (1 << 9, 2), 8))
        assert "below threshold" in str(e.value)
        m = rand_field(Z.BABYBEAR, (1 << 10, 2), 9)
        assert (dft.dft_batch(m) == oracle.dft_batch(Z.BABYBEAR, m)).all()
    finally:
        N.set_thresholds()
