"""Device-resident Pauli sum and propagation through the C ABI (pl_state_*).

Mirrors the reference's PauliSum methods that the propagation loop uses
(evolve, canonicalize, sort_and_combine, cutoff, truncate_weight,
apply_CNOT, zero_state_expectation; PauliSumOperations.h / PauliSumUtils.h)
and the driver (propagate / propagate_expectation, PauliPropagation.h:54-71).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

U64_MAX = (1 << 64) - 1


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


def truncation(max_weight=None, cutoff=0.0, max_terms=None) -> _abi.Truncation:
    return _abi.Truncation(U64_MAX if max_weight is None else int(max_weight),
                           float(cutoff or 0.0), U64_MAX if max_terms is None else int(max_terms))


class State:
    """A Pauli sum kept on the GPU between gates (``pl_state``)."""

    def __init__(self, array_size: int, capacity_hint: int = 1 << 16, stream=None):
        self.array_size = int(array_size)
        self._lib = _abi.lib()
        h = C.c_void_p()
        s = stream if stream is not None else _default_stream()
        _abi.check(self._lib.pl_state_create(C.byref(h), self.array_size, int(capacity_hint), s),
                   "pl_state_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pl_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def use_graphs(self, enable: bool = True):
        """Replay runs of single-qubit rotations from captured CUDA graphs."""
        _abi.check(self._lib.pl_state_set_option(self._h, _abi.PL_OPT_GRAPHS, int(bool(enable))),
                   "pl_state_set_option")
        return self

    def set_cancel_flag(self, flag: "np.ndarray | None"):
        """Stop propagate() between gates (PL_ERR_CANCELLED) once flag[0]
        (an int32 array the caller keeps alive) becomes non-zero; None
        clears it."""
        self._cancel = flag
        p = None if flag is None else flag.ctypes.data_as(C.c_void_p)
        _abi.check(self._lib.pl_state_set_cancel_flag(self._h, p), "pl_state_set_cancel_flag")
        return self

    # -- sharded sums (pl_state_shard_pack / _unpack, MpiPauliSum.h) -------
    def shard_pack(self, ranks: int):
        """This state's terms as (n, 2*AS + 2) int64 records on the device,
        grouped by owner rank FNV-1a(x, z) mod ranks in term order, and the
        per-owner counts."""
        import torch
        n = self.size()
        W = 2 * self.array_size + 2
        recs = torch.empty((max(n, 1), W), dtype=torch.int64, device="cuda")
        counts = (C.c_int64 * int(ranks))()
        _abi.check(self._lib.pl_state_shard_pack(self._h, int(ranks), recs.data_ptr(), n,
                                                 counts), "pl_state_shard_pack")
        return recs, [int(c) for c in counts]

    def shard_unpack(self, recs):
        """Replace the terms by the records received (an (m, W) tensor)."""
        m = int(recs.shape[0])
        _abi.check(self._lib.pl_state_shard_unpack(self._h, recs.data_ptr() if m else None, m),
                   "pl_state_shard_unpack")

    def max_abs(self) -> float:
        r = C.c_double()
        _abi.check(self._lib.pl_state_max_abs(self._h, C.byref(r)), "pl_state_max_abs")
        return r.value

    def count_above(self, threshold: float) -> int:
        c = C.c_int64()
        _abi.check(self._lib.pl_state_count_above(self._h, float(threshold), C.byref(c)),
                   "pl_state_count_above")
        return int(c.value)

    def log_gates(self, enable: bool = True):
        """Record (terms in, anticommuting terms, terms out) of every
        fast-path rotation of the next propagate() (PL_OPT_GATE_LOG)."""
        _abi.check(self._lib.pl_state_set_option(self._h, _abi.PL_OPT_GATE_LOG,
                                                 int(bool(enable))), "pl_state_set_option")
        return self

    def gate_log(self) -> np.ndarray:
        """(ops, 3) int64 sizes of the last propagate(), in processing order
        (the circuit reversed); rows of ops that are not fast-path rotations
        are zero."""
        n = C.c_int64()
        _abi.check(self._lib.pl_state_gate_log(self._h, None, 0, C.byref(n)), "pl_state_gate_log")
        out = np.zeros((n.value, 3), np.int64)
        if n.value:
            _abi.check(self._lib.pl_state_gate_log(self._h, out.ctypes.data_as(C.c_void_p),
                                                   n.value, C.byref(n)), "pl_state_gate_log")
        return out

    def memory(self) -> int:
        b = C.c_uint64()
        _abi.check(self._lib.pl_state_memory(self._h, C.byref(b)), "pl_state_memory")
        return b.value

    # -- data ------------------------------------------------------------
    def upload(self, x, z, flags, val):
        x = np.ascontiguousarray(x, np.uint64).reshape(self.array_size, -1)
        z = np.ascontiguousarray(z, np.uint64).reshape(self.array_size, -1)
        f = np.ascontiguousarray(flags, np.uint8)
        v = np.ascontiguousarray(val, np.float64)
        _abi.check(self._lib.pl_state_upload(self._h, _ptr(x), _ptr(z), _ptr(f), _ptr(v),
                                             v.shape[0]), "pl_state_upload")
        return self

    def size(self) -> int:
        n = C.c_int64()
        _abi.check(self._lib.pl_state_size(self._h, C.byref(n)), "pl_state_size")
        return n.value

    def download(self):
        n = self.size()
        x = np.zeros((self.array_size, n), np.uint64)
        z = np.zeros((self.array_size, n), np.uint64)
        f = np.zeros(n, np.uint8)
        v = np.zeros(n, np.float64)
        got = C.c_int64()
        if n:
            _abi.check(self._lib.pl_state_download(self._h, _ptr(x), _ptr(z), _ptr(f), _ptr(v),
                                                   n, C.byref(got)), "pl_state_download")
        return x, z, f, v

    # -- operations --------------------------------------------------------
    def evolve(self, rx, rz, rf, theta):
        rx = np.ascontiguousarray(rx, np.uint64).reshape(self.array_size, -1)
        rz = np.ascontiguousarray(rz, np.uint64).reshape(self.array_size, -1)
        rf = np.ascontiguousarray(rf, np.uint8)
        th = np.ascontiguousarray(theta, np.float64)
        _abi.check(self._lib.pl_state_evolve(self._h, _ptr(rx), _ptr(rz), _ptr(rf), _ptr(th),
                                             th.shape[0]), "pl_state_evolve")

    def apply_truncation(self, max_weight=None, cutoff=0.0, max_terms=None):
        t = truncation(max_weight, cutoff, max_terms)
        _abi.check(self._lib.pl_state_apply_truncation(self._h, C.byref(t)),
                   "pl_state_apply_truncation")

    def canonicalize(self):
        _abi.check(self._lib.pl_state_canonicalize(self._h), "pl_state_canonicalize")

    def sort_and_combine(self):
        _abi.check(self._lib.pl_state_sort_and_combine(self._h), "pl_state_sort_and_combine")

    def cutoff(self, eps):
        _abi.check(self._lib.pl_state_cutoff(self._h, float(eps)), "pl_state_cutoff")

    def truncate_weight(self, w):
        _abi.check(self._lib.pl_state_truncate_weight(self._h, int(w)), "pl_state_truncate_weight")

    def trim(self, max_terms, keep: "State | None" = None):
        if keep is None:
            _abi.check(self._lib.pl_state_trim(self._h, int(max_terms)), "pl_state_trim")
        else:
            _abi.check(self._lib.pl_state_trim_protected(self._h, int(max_terms), keep._h),
                       "pl_state_trim_protected")

    # -- reductions (PauliSumUtils.h:178-268, 400-447) --------------------
    def _scalar(self, fn, *args, what=""):
        r = C.c_double()
        _abi.check(fn(self._h, *args, C.byref(r)), what)
        return r.value

    def basis_state_expectation(self, bit_words):
        w = np.ascontiguousarray(bit_words, np.uint64)
        return self._scalar(self._lib.pl_state_basis_state_expectation, _ptr(w),
                            what="pl_state_basis_state_expectation")

    def trace(self, num_qubits):
        return self._scalar(self._lib.pl_state_trace, int(num_qubits), what="pl_state_trace")

    def frobenius_norm2(self):
        return self._scalar(self._lib.pl_state_frobenius_norm2, what="pl_state_frobenius_norm2")

    def lookup(self, x_words, z_words, flags):
        x = np.ascontiguousarray(x_words, np.uint64)
        z = np.ascontiguousarray(z_words, np.uint64)
        return self._scalar(self._lib.pl_state_lookup, _ptr(x), _ptr(z), int(flags) & 3,
                            what="pl_state_lookup")

    def trace_product(self, other: "State", num_qubits):
        return self._scalar(self._lib.pl_state_trace_product, other._h, int(num_qubits),
                            what="pl_state_trace_product")

    def apply_clifford(self, gate, q1, q2=0):
        """Bulk Clifford gate (name from _abi.GATES or its PL_GATE_* number)."""
        g = _abi.GATES[gate] if isinstance(gate, str) else int(gate)
        _abi.check(self._lib.pl_state_apply_clifford(self._h, g, int(q1), int(q2)),
                   "pl_state_apply_clifford")

    def apply_rotation_gate(self, axis, qubit, angle):
        """apply_RX / RY / RZ: axis "X"/"Y"/"Z" (or 1/2/3), exp(-i angle/2 P)."""
        a = {"X": 1, "Y": 2, "Z": 3}.get(axis, axis)
        _abi.check(self._lib.pl_state_apply_rotation_gate(self._h, int(a), int(qubit),
                                                          float(angle)),
                   "pl_state_apply_rotation_gate")

    def apply_cnot(self, c, t):
        _abi.check(self._lib.pl_state_apply_cnot(self._h, int(c), int(t)), "pl_state_apply_cnot")

    def zero_state_expectation(self) -> float:
        r = C.c_double()
        _abi.check(self._lib.pl_state_zero_state_expectation(self._h, C.byref(r)),
                   "pl_state_zero_state_expectation")
        return r.value

    def propagate(self, rx, rz, rf, theta, ops=None, max_weight=None, cutoff=0.0,
                  max_terms=None):
        rx = np.ascontiguousarray(rx, np.uint64).reshape(self.array_size, -1)
        rz = np.ascontiguousarray(rz, np.uint64).reshape(self.array_size, -1)
        rf = np.ascontiguousarray(rf, np.uint8)
        th = np.ascontiguousarray(theta, np.float64)
        t = truncation(max_weight, cutoff, max_terms)
        if ops is None:
            o, n_ops = None, 0
        else:
            o = np.ascontiguousarray(ops, np.int32).reshape(-1, 3)
            n_ops = o.shape[0]
        _abi.check(self._lib.pl_propagate(self._h, _ptr(rx), _ptr(rz), _ptr(rf), _ptr(th),
                                          th.shape[0], _ptr(o) if o is not None else None, n_ops,
                                          C.byref(t)), "pl_propagate")


def _default_stream():
    try:
        import torch
        if torch.cuda.is_available():
            return int(torch.cuda.current_stream().cuda_stream)
    except Exception:
        pass
    return None


def propagate_expectation_planes(obs, circ, max_weight=None, cutoff=0.0, max_terms=None,
                                 capacity_hint: int = 1 << 16) -> float:
    """<0|U^dagger O U|0> for a workloads.Circuit (rotations + CNOTs)."""
    with State(obs.x.shape[0], capacity_hint) as st:
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, max_weight, cutoff, max_terms)
        return st.zero_state_expectation()
