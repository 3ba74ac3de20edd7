"""ctypes binding of libzkb200.so (the C ABI declared in include/zkb200.h).

The shared library is built in-tree (``ziros_b200/libzkb200.so``).  Importing
this module never falls back to anything: a missing or unloadable library raises
``ZkbError`` so a GPU run can not silently take another path.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzkb200.so")

OK = 0
DECLINED = 1
ERR_INVALID = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_UNSUPPORTED = -4
ERR_INTERNAL = -5
ERR_TIMEOUT = -6
ERR_CANCELLED = -7

FIELD_BABYBEAR = 0
FIELD_GOLDILOCKS = 1


class ZkbError(RuntimeError):
    """A failed library call; `code` is the C status, the message is zkb_last_error_message()."""

    def __init__(self, code: int, message: str):
        super().__init__(f"zkb200 error {code}: {message}")
        self.code = code


class ZkbDeclined(ZkbError):
    """The library declined the call (reference `false`/`None`: use the CPU path)."""


class Matrix(C.Structure):
    _fields_ = [("data", C.c_void_p), ("height", C.c_uint64), ("width", C.c_uint64)]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_uint64), ("total_ms", C.c_double),
                ("max_ms", C.c_double)]


class Hasher(C.Structure):
    _fields_ = [("field", C.c_int), ("width", C.c_uint32), ("seed", C.c_uint64)]


class FriParams(C.Structure):
    _fields_ = [("log_n", C.c_uint32), ("log_final", C.c_uint32), ("challenge_seed", C.c_uint64),
                ("num_queries", C.c_uint32), ("query_seed", C.c_uint64), ("transcript", C.c_uint32)]


class EngineConfig(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("hbm_budget", C.c_uint64), ("policy", C.c_uint32)]


ADMIT_FIFO, ADMIT_SMALLEST, ADMIT_MAX_BYPASS = 0, 1, 8


class JobDesc(C.Structure):
    _fields_ = [("hasher", Hasher), ("trace", C.c_void_p), ("log_h", C.c_uint32), ("width", C.c_uint32),
                ("log_blowup", C.c_uint32), ("with_fri", C.c_int), ("alpha", C.c_uint32 * 4),
                ("fri", FriParams)]


class JobResult(C.Structure):
    _fields_ = [("status", C.c_int), ("root", C.c_uint32 * 16), ("queue_ms", C.c_double),
                ("run_ms", C.c_double), ("latency_ms", C.c_double)]


class RtNode(C.Structure):
    _fields_ = [("kind", C.c_int), ("field", C.c_int), ("log_n", C.c_uint32), ("width", C.c_uint32),
                ("log_blowup", C.c_uint32), ("inverse", C.c_uint32), ("count", C.c_uint64), ("in_slot", C.c_int),
                ("out_slot", C.c_int), ("seed", C.c_uint64), ("hasher_width", C.c_uint32), ("ext4", C.c_uint32),
                ("beta", C.c_uint32 * 4), ("tree_node", C.c_int)]


class Thresholds(C.Structure):
    _fields_ = [("ntt", C.c_uint64), ("poseidon2", C.c_uint64), ("merkle", C.c_uint64), ("fri", C.c_uint64)]


class BatchShape(C.Structure):
    _fields_ = [("log_h", C.c_uint32), ("width", C.c_uint32)]


class BatchOptions(C.Structure):
    _fields_ = [("log_blowup", C.c_uint32), ("use_graph", C.c_int), ("branches", C.c_uint32),
                ("autotune", C.c_int), ("tune_cache", C.c_char_p)]


class BatchInfo(C.Structure):
    _fields_ = [("device_bytes", C.c_uint64), ("kernels_per_run", C.c_uint32), ("branches", C.c_uint32),
                ("leaf_threads", C.c_uint32), ("use_graph", C.c_int), ("tuned_from_cache", C.c_int),
                ("tune_ms", C.c_double)]


class BatchQueueInfo(C.Structure):
    _fields_ = [("items", C.c_uint32), ("steps", C.c_uint32), ("stages", C.c_uint32), ("grid", C.c_uint32),
                ("leaf_levels", C.c_uint32), ("comp_levels", C.c_uint32)]


class EngineStats(C.Structure):
    _fields_ = [("queued", C.c_uint64), ("completed", C.c_uint64), ("hbm_budget", C.c_uint64),
                ("hbm_in_use", C.c_uint64), ("hbm_peak", C.c_uint64)]


# Every symbol of include/zkb200.h with its ctypes signature.
_P = C.c_void_p
_SZ = C.c_size_t
_U32 = C.c_uint32
_U64 = C.c_uint64
_I = C.c_int
SIGNATURES = {
    "zkb_version": (C.c_char_p, []),
    "zkb_last_error_message": (C.c_char_p, []),
    "zkb_device_count": (_I, []),
    "zkb_set_device": (_I, [_I]),
    "zkb_measure_mul_peak": (_I, [_I, _P]),
    "zkb_profile_start": (_I, []),
    "zkb_profile_stop": (_I, [_P, _I]),
    "zkb_poseidon2_babybear_round_constants": (_I, [_U64, _P, _SZ, _P, _P]),
    "zkb_poseidon2_goldilocks_round_constants": (_I, [_U64, _U32, _P, _SZ, _P, _P]),
    "zkb_poseidon2_babybear_permute": (_I, [_P, _SZ, _P, _SZ, _U32, _U32]),
    "zkb_poseidon2_goldilocks_permute": (_I, [_P, _SZ, _P, _SZ, _U32, _U32]),
    "zkb_poseidon2_babybear_permute_dev": (_I, [_P, _SZ, _P, _SZ, _U32, _U32, _P]),
    "zkb_poseidon2_goldilocks_permute_dev": (_I, [_P, _SZ, _P, _SZ, _U32, _U32, _P]),
    "zkb_dft_batch": (_I, [_I, _P, _U32, _U32, _I]),
    "zkb_dft_batch_dev": (_I, [_I, _P, _U32, _U32, _I, _P]),
    "zkb_dft_batch_noalloc_dev": (_I, [_I, _P, _U32, _U32, _I, _P]),
    "zkb_set_ntt_tile_loads": (_I, [_I]),
    "zkb_ntt_tile_load_errors": (_I, [_P]),
    "zkb_coset_lde_batch": (_I, [_I, _P, _U32, _U32, _U32, _U64, _I, _P]),
    "zkb_coset_lde_batch_dev": (_I, [_I, _P, _U32, _U32, _U32, _U64, _I, _P, _P]),
    "zkb_mmcs_commit": (_I, [_P, _P, _SZ, _P, _P]),
    "zkb_mmcs_commit_dev": (_I, [_P, _P, _SZ, _P, _P, _P]),
    "zkb_pcs_commit": (_I, [_P, _P, _U32, _U32, _U32, _P, _P]),
    "zkb_pcs_commit_dev": (_I, [_P, _P, _U32, _U32, _U32, _P, _P, _P]),
    "zkb_tree_matrix_dev": (_P, [_P, _I]),
    "zkb_tree_num_layers": (_I, [_P]),
    "zkb_tree_layer_len": (C.c_int64, [_P, _I]),
    "zkb_tree_digest_elems": (_I, [_P]),
    "zkb_tree_copy_layer": (_I, [_P, _I, _P]),
    "zkb_mmcs_open_batch": (_I, [_P, _U64, _P, _SZ, _P, _SZ]),
    "zkb_tree_free": (None, [_P]),
    "zkb_fri_fold_goldilocks": (_I, [_P, _SZ, _U64, _P, _P]),
    "zkb_fri_fold_babybear": (_I, [_P, _SZ, _U32, _P, _P]),
    "zkb_fri_fold_babybear_ext4": (_I, [_P, _SZ, _P, _P]),
    "zkb_fri_commit_babybear_ext4": (_I, [_P, _P, _P, _P]),
    "zkb_fri_commit_babybear_ext4_dev": (_I, [_P, _P, _P, _P, _P]),
    "zkb_fri_num_rounds": (_I, [_P]),
    "zkb_fri_commitments": (_I, [_P, _P, _P]),
    "zkb_fri_final_codeword": (_I, [_P, _P]),
    "zkb_fri_siblings_per_query": (C.c_int64, [_P]),
    "zkb_fri_query_openings": (_I, [_P, _P, _P, _P]),
    "zkb_fri_proof_free": (None, [_P]),
    "zkb_combine_columns_babybear_ext4_dev": (_I, [_P, _U64, _U32, _P, _P, _P]),
    "zkb_pcs_commit_fri": (_I, [_P, _P, _U32, _U32, _U32, _P, _P, _P, _P, _P]),
    "zkb_engine_create": (_I, [_P, _P]),
    "zkb_engine_submit": (_I, [_P, _P, _P]),
    "zkb_engine_wait": (_I, [_P, _U64, _P, _P]),
    "zkb_engine_stats": (_I, [_P, _P]),
    "zkb_engine_destroy": (None, [_P]),
    "zkb_coset_lde_tuned_dev": (_I, [_I, _P, _U32, _U32, _U32, _I, _U32, _U32, _P, _P]),
    "zkb_fri_alpha": (_I, [_P, _P]),
    "zkb_poly_eval_goldilocks": (_I, [_P, _SZ, _P, _SZ, _P]),
    "zkb_poly_coset_eval_goldilocks": (_I, [_P, _U32, _U64, _P]),
    "zkb_poly_quotient_goldilocks": (_I, [_P, _U32, _U64, _U64, _P]),
    "zkb_rt_create": (_I, [_P]),
    "zkb_rt_buffer": (_I, [_P, _U64, _P]),
    "zkb_rt_write": (_I, [_P, _I, _P, _U64]),
    "zkb_rt_read": (_I, [_P, _I, _P, _U64]),
    "zkb_rt_add": (_I, [_P, _P, _P, _SZ, _P]),
    "zkb_rt_execute": (_I, [_P, _P, _P]),
    "zkb_rt_node_ms": (_I, [_P, _I, _P]),
    "zkb_rt_tree": (_I, [_P, _I, _P]),
    "zkb_rt_free": (None, [_P]),
    "zkb_set_thresholds": (_I, [_P]),
    "zkb_get_thresholds": (_I, [_P]),
    "zkb_circuit_open": (_I, [C.c_char_p, _SZ]),
    "zkb_circuit_reset": (None, []),
    "zkb_debug_inject_fault": (_I, [_I, _I]),
    "zkb_batch_set_merkle_fusion": (_I, [_P, _U32, _U32]),
    "zkb_batch_queue_info": (_I, [_P, _P]),
    "zkb_batch_profile": (_I, [_P, _P, _P, _P]),
    "zkb_debug_batch_stalled_run": (_I, [_P, _U64, _P]),
    "zkb_debug_device_allocations": (_U64, []),
    "zkb_debug_pool_allocations": (_U64, []),
    "zkb_release_cached_memory": (_I, []),
    "zkb_engine_cancel": (_I, [_P, _U64]),
    "zkb_mmcs_verify_batch": (_I, [_P, _P, _P, _P, _SZ, _U64, _P, _P, _SZ]),
    "zkb_challenger_create": (_I, [_P, _P]),
    "zkb_challenger_observe": (_I, [_P, _P, _SZ]),
    "zkb_challenger_sample": (_I, [_P, _P, _SZ]),
    "zkb_challenger_sample_bits": (_I, [_P, _U32, _P]),
    "zkb_challenger_free": (None, [_P]),
    "zkb_fri_commit_babybear_ext4_challenger_dev": (_I, [_P, _P, _P, _P, _P, _P]),
    "zkb_mmcs_compress": (_I, [_P, _P, _P, _SZ, _P]),
    "zkb_mmcs_commit_reduce_dev": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "zkb_batch_create": (_I, [_P, _P, _SZ, _P, _P]),
    "zkb_batch_trace_ptr": (_I, [_P, _SZ, _P]),
    "zkb_batch_copy_in": (_I, [_P, _SZ, _P, _I, _P]),
    "zkb_batch_run": (_I, [_P, _P]),
    "zkb_batch_run_host": (_I, [_P, _P, _P]),
    "zkb_batch_roots": (_I, [_P, _P, _P]),
    "zkb_batch_tree": (_I, [_P, _SZ, _P]),
    "zkb_batch_info": (_I, [_P, _P]),
    "zkb_batch_lde_tune": (_I, [_P, _SZ, _P, _P, _P]),
    "zkb_batch_free": (None, [_P]),
    "zkb_pcs_commit_fri_dev": (_I, [_P, _P, _U32, _U32, _U32, _P, _P, _P, _P, _P, _P]),
}

_lib = None
_lock = threading.Lock()


def load():
    """Load libzkb200.so (raises ZkbError if it is missing or incomplete)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ZkbError(ERR_INTERNAL, f"{LIB_PATH} is not built (run ziros_b200.build.build())")
        try:
            lib = C.CDLL(LIB_PATH)
        except OSError as e:  # pragma: no cover - depends on the environment
            raise ZkbError(ERR_INTERNAL, f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def circuit_open() -> tuple:
    """(open, reason) of the library's failure circuit."""
    buf = C.create_string_buffer(512)
    return bool(load().zkb_circuit_open(buf, 512)), buf.value.decode(errors="replace")


def set_thresholds(ntt: int = 0, poseidon2: int = 0, merkle: int = 0, fri: int = 0) -> None:
    """Minimum sizes below which host-pointer calls decline (all 0: never)."""
    check(load().zkb_set_thresholds(C.byref(Thresholds(ntt, poseidon2, merkle, fri))))


def get_thresholds() -> dict:
    t = Thresholds()
    check(load().zkb_get_thresholds(C.byref(t)))
    return {k: int(getattr(t, k)) for k, _ in Thresholds._fields_}


def circuit_reset() -> None:
    load().zkb_circuit_reset()


def inject_fault(kind: int, count: int = 1) -> None:
    """Host-side fault injection for tests (1: allocations fail, 2: waits time out)."""
    check(load().zkb_debug_inject_fault(kind, count))


def device_allocations() -> int:
    """Device allocations the library has made in this process (pool or cudaMalloc)."""
    return int(load().zkb_debug_device_allocations())


def pool_allocations() -> int:
    """Device allocations of 1 MiB or more that missed the library's block cache (new pool memory)."""
    return int(load().zkb_debug_pool_allocations())


def release_cached_memory() -> None:
    """Returns the library's cached device blocks and the pool's unused memory to the device."""
    check(load().zkb_release_cached_memory())


def set_ntt_tile_loads(mode: int) -> None:
    """NTT tiles: 1 = one tensor copy per tile (default), 0 = coalesced loads into registers."""
    check(load().zkb_set_ntt_tile_loads(int(mode)))


def ntt_tile_load_errors() -> int:
    """Tensor-copy waits of the NTT passes that gave up since the last call (resets)."""
    n = C.c_uint32(0)
    check(load().zkb_ntt_tile_load_errors(C.byref(n)))
    return n.value


def last_error() -> str:
    msg = load().zkb_last_error_message()
    return msg.decode() if msg else ""


def check(rc: int) -> int:
    """Raise on a negative status; DECLINED raises ZkbDeclined."""
    if rc == OK or rc > DECLINED:
        return rc
    if rc == DECLINED:
        raise ZkbDeclined(rc, last_error())
    raise ZkbError(rc, last_error())


def profile_start() -> None:
    check(load().zkb_profile_start())


def profile_stop() -> dict:
    """{kernel name: (launches, total_ms, max_ms)} since profile_start()."""
    buf = (KernelStat * 64)()
    n = load().zkb_profile_stop(buf, 64)
    check(n if n < 0 else 0)
    return {buf[i].name.decode(): (int(buf[i].launches), float(buf[i].total_ms), float(buf[i].max_ms))
            for i in range(min(n, 64))}


def measure_mul_peak(field: int) -> float:
    """Field multiplications per second of the device's multiply pipe (see diag.cu)."""
    v = C.c_double()
    check(load().zkb_measure_mul_peak(field, C.byref(v)))
    return float(v.value)


def device_count() -> int:
    return int(load().zkb_device_count())
