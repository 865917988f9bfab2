"""ctypes binding of the C ABI in include/paulib_b200.h.

The shared library is built in-tree (``python -m paulib_b200.build``); if it
is missing this module raises -- there is no CPU fallback.  Device buffers
are torch tensors (plumbing only: allocation, copies, streams).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpaulib_b200.so")

VP = C.c_void_p
I64 = C.c_int64
I32 = C.c_int

PL_OK = 0
PL_ERR_INVALID_ARG = 1
PL_ERR_OOM = 2
PL_ERR_TIMEOUT = 3
PL_ERR_CUDA = 4
PL_ERR_CAPACITY = 5
PL_ERR_UNSUPPORTED = 6
PL_ERR_INTERNAL = 7
PL_ERR_CANCELLED = 8
PL_COLLATE_CANONICALIZE = 0
PL_COLLATE_SORT_AND_COMBINE = 1
UINT64_MAX = (1 << 64) - 1

# Every symbol include/paulib_b200.h declares.
EXPORTS = (
    "pl_status_string", "pl_get_last_error", "pl_last_error_message", "pl_version",
    "launch_gpu_mul_soa", "launch_gpu_commutator_soa", "pl_multiply", "pl_commutator",
    "pl_collate_workspace_size", "pl_collate", "pl_multiply_collate_workspace_size",
    "pl_multiply_collate", "pl_apply_cnot", "pl_zero_state_expectation",
    "pl_state_create", "pl_state_destroy", "pl_state_upload", "pl_state_download",
    "pl_state_size", "pl_state_evolve", "pl_state_apply_truncation", "pl_state_canonicalize",
    "pl_state_sort_and_combine", "pl_state_cutoff", "pl_state_truncate_weight",
    "pl_state_apply_cnot", "pl_state_zero_state_expectation", "pl_propagate",
    "pl_profile_reset", "pl_profile_read", "pl_state_multiply",
    "pl_state_multiply_canonicalize", "pl_state_commutator", "pl_profile_report",
    "pl_commutator_noalloc", "pl_state_set_option", "pl_state_memory", "pl_batch_propagate",
    "pl_serve", "pl_state_trim", "pl_state_trim_protected", "pl_state_append",
    "pl_set_tuning", "pl_get_tuning", "pl_state_apply_clifford", "pl_state_apply_rotation_gate",
    "pl_state_basis_state_expectation", "pl_state_trace", "pl_state_frobenius_norm2",
    "pl_state_lookup", "pl_state_trace_product", "pl_state_shard_pack", "pl_state_shard_unpack",
    "pl_state_count_above", "pl_state_max_abs", "pl_state_gate_log", "pl_job_estimate",
    "pl_state_set_cancel_flag", "pl_check_bounded_wait",
)
PL_OP_CLIFFORD = 100
GATES = {"H": 1, "S": 2, "H_YZ": 3, "H_XY": 4, "SQRT_X": 5, "SQRT_Y": 6, "X": 7, "Y": 8,
         "Z": 9, "I": 10, "CNOT": 11, "CZ": 12, "CY": 13, "XC_X": 14, "XC_Y": 15, "XC_Z": 16,
         "YC_X": 17, "YC_Y": 18, "YC_Z": 19, "SWAP": 20, "ISWAP": 21}
PL_TUNE_RADIX_ITEMS = 1
PL_TUNE_INDEX_KEYS = 2
PL_TUNE_SPIN_LIMIT = 3
PL_TUNE_FAIL_ALLOC = 4
PL_TUNE_WINDOW_KEYS = 5
PL_TUNE_RADIX_PREFETCH = 6
PL_TUNE_RADIX_WINDOW = 7
PL_TUNE_RADIX_WIDE = 8
PL_TUNE_RADIX_BACKOFF = 9
PL_TUNE_FOLD_GATHER = 10
PL_OPT_GRAPHS = 1
PL_OPT_GATE_LOG = 2
PL_ORDER_GIVEN = 0
PL_ORDER_LONGEST_FIRST = 1


class CollateOpts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("reserved", C.c_int32), ("cutoff", C.c_double),
                ("max_weight", C.c_uint64)]


class Truncation(C.Structure):
    _fields_ = [("max_weight", C.c_uint64), ("coefficient_cutoff", C.c_double),
                ("max_terms", C.c_uint64)]


class Job(C.Structure):
    _fields_ = [("array_size", C.c_int32), ("obs_x", VP), ("obs_z", VP), ("obs_flags", VP),
                ("obs_val", VP), ("obs_n", I64), ("rot_x", VP), ("rot_z", VP),
                ("rot_flags", VP), ("rot_theta", VP), ("n_rot", I64), ("ops", VP),
                ("n_ops", I64), ("trunc", Truncation), ("arrival_s", C.c_double),
                ("cancel", VP)]


class JobResult(C.Structure):
    _fields_ = [("expectation", C.c_double), ("final_terms", I64), ("status", C.c_int32),
                ("lane", C.c_int32), ("start_s", C.c_double), ("end_s", C.c_double)]


class BatchOpts(C.Structure):
    _fields_ = [("lanes", C.c_int32), ("use_graphs", C.c_int32), ("order", C.c_int32),
                ("hbm_budget", C.c_uint64), ("keep_bytes", C.c_uint64), ("sync_stream", VP)]


class BatchStats(C.Structure):
    _fields_ = [("wall_s", C.c_double), ("peak_bytes", C.c_uint64),
                ("budget_waits", C.c_uint64), ("jobs_failed", C.c_uint64),
                ("jobs_rejected", C.c_uint64), ("admission_waits", C.c_uint64)]


class PLError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib = None


def lib():
    """Load libpaulib_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m paulib_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.pl_status_string.restype = C.c_char_p
    L.pl_status_string.argtypes = [I32]
    L.pl_last_error_message.restype = C.c_char_p
    L.pl_get_last_error.restype = I32
    L.pl_version.restype = I32
    sig = {
        "launch_gpu_mul_soa": (None, [I32] + [VP] * 12 + [I32, I32, VP]),
        "launch_gpu_commutator_soa": (None, [I32, I32] + [VP] * 13 + [I32, I32, C.c_longlong,
                                                                      VP]),
        "pl_multiply": (I32, [I32, VP, VP, VP, VP, I64, VP, VP, VP, VP, I64, VP, VP, VP, VP,
                              VP]),
        "pl_commutator": (I32, [I32, I32, VP, VP, VP, VP, I64, VP, VP, VP, VP, I64, VP, VP,
                                VP, VP, I64, VP, VP]),
        "pl_commutator_noalloc": (I32, [I32, I32, VP, VP, VP, VP, I64, VP, VP, VP, VP, I64, VP,
                                        VP, VP, VP, I64, VP, VP]),
        "pl_collate_workspace_size": (I32, [I32, I64, C.POINTER(C.c_size_t)]),
        "pl_collate": (I32, [I32, VP, VP, VP, VP, I64, VP, VP, VP, VP, I64, C.POINTER(I64),
                             C.POINTER(CollateOpts), VP, C.c_size_t, VP]),
        "pl_multiply_collate_workspace_size": (I32, [I32, I64, I64, C.POINTER(C.c_size_t)]),
        "pl_multiply_collate": (I32, [I32, VP, VP, VP, VP, I64, VP, VP, VP, VP, I64, VP, VP,
                                      VP, VP, I64, C.POINTER(I64), C.POINTER(CollateOpts), VP,
                                      C.c_size_t, VP]),
        "pl_apply_cnot": (I32, [I32, VP, VP, VP, I64, I64, I32, I32, VP]),
        "pl_zero_state_expectation": (I32, [I32, VP, VP, VP, I64, I64, VP, VP]),
        "pl_state_create": (I32, [C.POINTER(VP), I32, I64, VP]),
        "pl_state_destroy": (I32, [VP]),
        "pl_state_upload": (I32, [VP, VP, VP, VP, VP, I64]),
        "pl_state_download": (I32, [VP, VP, VP, VP, VP, I64, C.POINTER(I64)]),
        "pl_state_size": (I32, [VP, C.POINTER(I64)]),
        "pl_state_evolve": (I32, [VP, VP, VP, VP, VP, I64]),
        "pl_state_apply_truncation": (I32, [VP, C.POINTER(Truncation)]),
        "pl_state_canonicalize": (I32, [VP]),
        "pl_state_sort_and_combine": (I32, [VP]),
        "pl_state_cutoff": (I32, [VP, C.c_double]),
        "pl_state_truncate_weight": (I32, [VP, C.c_uint64]),
        "pl_state_apply_cnot": (I32, [VP, I32, I32]),
        "pl_state_zero_state_expectation": (I32, [VP, C.POINTER(C.c_double)]),
        "pl_propagate": (I32, [VP, VP, VP, VP, VP, I64, VP, I64, C.POINTER(Truncation)]),
        "pl_profile_reset": (I32, [I32]),
        "pl_profile_report": (I32, [C.c_char_p, C.c_size_t]),
        "pl_state_multiply": (I32, [VP, VP]),
        "pl_state_multiply_canonicalize": (I32, [VP, VP]),
        "pl_state_commutator": (I32, [VP, VP, VP, I32]),
        "pl_state_set_option": (I32, [VP, I32, I64]),
        "pl_state_trim": (I32, [VP, C.c_uint64]),
        "pl_state_append": (I32, [VP, VP]),
        "pl_state_apply_clifford": (I32, [VP, I32, I32, I32]),
        "pl_state_basis_state_expectation": (I32, [VP, VP, C.POINTER(C.c_double)]),
        "pl_state_trace": (I32, [VP, I32, C.POINTER(C.c_double)]),
        "pl_state_frobenius_norm2": (I32, [VP, C.POINTER(C.c_double)]),
        "pl_state_lookup": (I32, [VP, VP, VP, C.c_uint8, C.POINTER(C.c_double)]),
        "pl_state_trace_product": (I32, [VP, VP, I32, C.POINTER(C.c_double)]),
        "pl_state_shard_pack": (I32, [VP, I32, VP, I64, C.POINTER(I64)]),
        "pl_state_shard_unpack": (I32, [VP, VP, I64]),
        "pl_state_count_above": (I32, [VP, C.c_double, C.POINTER(I64)]),
        "pl_state_max_abs": (I32, [VP, C.POINTER(C.c_double)]),
        "pl_state_gate_log": (I32, [VP, VP, I64, C.POINTER(I64)]),
        "pl_job_estimate": (I32, [C.POINTER(Job), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_uint64)]),
        "pl_state_set_cancel_flag": (I32, [VP, VP]),
        "pl_check_bounded_wait": (I32, [C.POINTER(C.c_int)]),
        "pl_state_apply_rotation_gate": (I32, [VP, I32, I32, C.c_double]),
        "pl_set_tuning": (I32, [I32, I64]),
        "pl_get_tuning": (I32, [I32, C.POINTER(I64)]),
        "pl_state_trim_protected": (I32, [VP, C.c_uint64, VP]),
        "pl_state_memory": (I32, [VP, C.POINTER(C.c_uint64)]),
        "pl_batch_propagate": (I32, [C.POINTER(Job), I64, C.POINTER(BatchOpts),
                                     C.POINTER(JobResult), C.POINTER(BatchStats)]),
        "pl_serve": (I32, [C.POINTER(Job), I64, C.POINTER(BatchOpts), C.POINTER(JobResult),
                           C.POINTER(BatchStats)]),
        "pl_profile_read": (I32, [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int, what: str = ""):
    if status != PL_OK:
        L = lib()
        msg = (L.pl_last_error_message() or b"").decode()
        raise PLError(status, f"{what}: {msg}" if what else msg)


def last_error() -> int:
    return int(lib().pl_get_last_error())


# ---------------------------------------------------------------------------
# Device buffers (torch as the allocator).
# ---------------------------------------------------------------------------
def _torch():
    import torch
    return torch


class DeviceSum:
    """SoA planes of a Pauli sum in device memory: x/z are (AS, capacity)."""

    def __init__(self, array_size: int, capacity: int, device="cuda"):
        torch = _torch()
        cap = max(int(capacity), 1)
        self.array_size = int(array_size)
        self.capacity = cap
        self.x = torch.zeros((array_size, cap), dtype=torch.int64, device=device)
        self.z = torch.zeros((array_size, cap), dtype=torch.int64, device=device)
        self.flags = torch.zeros(cap, dtype=torch.uint8, device=device)
        self.val = torch.zeros(cap, dtype=torch.float64, device=device)
        self.n = 0

    @classmethod
    def from_host(cls, x, z, flags, val, capacity=None, device="cuda"):
        torch = _torch()
        x = np.ascontiguousarray(x, np.uint64)
        n = int(np.asarray(val).shape[0])
        ds = cls(x.shape[0], capacity if capacity is not None else n, device)
        if n:
            ds.x[:, :n].copy_(torch.from_numpy(x.view(np.int64)))
            ds.z[:, :n].copy_(torch.from_numpy(np.ascontiguousarray(z, np.uint64).view(np.int64)))
            ds.flags[:n].copy_(torch.from_numpy(np.ascontiguousarray(flags, np.uint8)))
            ds.val[:n].copy_(torch.from_numpy(np.ascontiguousarray(val, np.float64)))
        ds.n = n
        return ds

    def ptrs(self):
        return (self.x.data_ptr(), self.z.data_ptr(), self.flags.data_ptr(), self.val.data_ptr())

    def to_host(self, n=None):
        n = self.n if n is None else int(n)
        x = self.x[:, :n].cpu().numpy().view(np.uint64).copy()
        z = self.z[:, :n].cpu().numpy().view(np.uint64).copy()
        return x, z, self.flags[:n].cpu().numpy().copy(), self.val[:n].cpu().numpy().copy()


def stream_ptr(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def workspace(nbytes: int, device="cuda"):
    torch = _torch()
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)


def profile_reset(timing: bool = False):
    check(lib().pl_profile_reset(int(bool(timing))), "pl_profile_reset")


def profile_read():
    """(launches, timed_launches, timed_ms, timed_bytes) since the last reset."""
    a, b, d = C.c_uint64(), C.c_uint64(), C.c_uint64()
    ms = C.c_double()
    check(lib().pl_profile_read(C.byref(a), C.byref(b), C.byref(ms), C.byref(d)),
          "pl_profile_read")
    return a.value, b.value, ms.value, d.value


def profile_report() -> dict:
    """{kernel name: (launches, total_ms, bytes)} of the timed launches."""
    buf = C.create_string_buffer(1 << 16)
    check(lib().pl_profile_report(buf, len(buf)), "pl_profile_report")
    out = {}
    for ln in buf.value.decode().splitlines():
        name, cnt, ms, nbytes = ln.split()
        out[name] = (int(cnt), float(ms), int(nbytes))
    return out
