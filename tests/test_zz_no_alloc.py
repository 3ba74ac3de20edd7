"""The allocation-free DFT entry point (zkb_dft_batch_noalloc_dev).

It exists for callers that cannot call cudaMalloc — a prover running inside a
process whose device memory is owned by another allocator, or a latency-critical
loop that must not pay the synchronisation of an allocation.  Its scratch is a
fixed device array inside the library, shared by every call, so this test calls it
twice in a row (with different inputs and shapes) and checks each result bit-exactly
against the allocating entry point zkb_dft_batch_dev.  It is collected last so a
failure here does not hide the other tests, and it passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import ziros_b200 as Z
from conftest import rand_field
from ziros_b200 import _native as N

pytestmark = pytest.mark.gpu


def _run(fn_name, field, host, inverse):
    import torch

    dt = torch.int32 if field == 0 else torch.int64
    t = torch.from_numpy(host.view(np.int32 if field == 0 else np.int64).copy()).cuda()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    fn = getattr(N.load(), fn_name)
    rc = fn(field, C.c_void_p(t.data_ptr()), host.shape[0].bit_length() - 1, host.shape[1], int(inverse), stream)
    N.check(rc)
    torch.cuda.synchronize()
    assert t.dtype == dt
    return t.cpu().numpy().view(host.dtype)


@pytest.mark.parametrize("field", [0, 1])
def test_noalloc_matches_allocating_entry_point_twice(field):
    cases = [((1 << 12, 16), False, 5), ((1 << 9, 3), True, 6)]
    for shape, inverse, seed in cases:  # two calls in a row share the fixed scratch
        m = rand_field(field, shape, seed)
        got = _run("zkb_dft_batch_noalloc_dev", field, m, inverse)
        want = _run("zkb_dft_batch_dev", field, m, inverse)
        assert (got == want).all()


@pytest.mark.parametrize("field", [0, 1])
def test_noalloc_makes_no_device_allocation(field):
    """The library counts every device allocation it makes; a shape no other call has
    used (so no cached table exists for it) must leave the count unchanged."""
    m = rand_field(field, (1 << 11, 5), 8)
    before = N.device_allocations()
    got = _run("zkb_dft_batch_noalloc_dev", field, m, True)
    assert N.device_allocations() == before
    assert (got == _run("zkb_dft_batch_dev", field, m, True)).all()
    assert N.device_allocations() > before  # the allocating entry point is counted


def test_noalloc_declines_while_circuit_open():
    """Like every entry point, it does no GPU work while the circuit is open."""
    import torch

    t = torch.zeros((1 << 6, 2), dtype=torch.int32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = N.load()
    N.inject_fault(2, 1)  # the next stream wait reports an expired deadline: the circuit opens
    try:
        with pytest.raises(N.ZkbError):
            Z.CudaDft(0).dft_batch(rand_field(0, (1 << 6, 2), 1))
        assert lib.zkb_dft_batch_noalloc_dev(0, C.c_void_p(t.data_ptr()), 6, 2, 0, stream) == N.DECLINED
        assert "circuit open" in N.last_error()
    finally:
        N.inject_fault(2, 0)
        N.circuit_reset()
    N.check(lib.zkb_dft_batch_noalloc_dev(0, C.c_void_p(t.data_ptr()), 6, 2, 0, stream))


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch

    t = torch.zeros((1 << 20, 8), dtype=torch.int32, device="cuda")
    rc = N.load().zkb_dft_batch_noalloc_dev(0, C.c_void_p(t.data_ptr()), 20, 8, 0,
                                            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == N.ERR_INVALID
    assert "fixed scratch" in N.last_error()
