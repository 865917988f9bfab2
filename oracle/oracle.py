"""ctypes access to the parity oracle -- TEST INFRASTRUCTURE ONLY.

Two CPU implementations of PauLIB's Pauli-sum hot path share one interface:

* ``Oracle``    -- the plain-C restatement in ``oracle/paulib_oracle.c``
                   (strict IEEE, single-threaded, sequential sums).
* ``Reference`` -- the reference's own header-only code compiled in place by
                   ``oracle/Makefile`` into ``oracle/_ref/`` (OpenMP, the
                   reference's -O3 -ffast-math flags).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg may
import this module, and only as the checker / CPU baseline.

A sum crosses the boundary as numpy SoA planes: ``x``/``z`` of shape
(AS, n) uint64, ``flags`` (n,) uint8, ``val`` (n,) float64.
"""
from __future__ import annotations

import ctypes as C
import os
import platform

import numpy as np

from paulib_b200.planes import Planes  # noqa: F401  (re-exported for the tests)

HERE = os.path.dirname(os.path.abspath(__file__))
U64P = C.POINTER(C.c_uint64)
U8P = C.POINTER(C.c_uint8)
F64P = C.POINTER(C.c_double)
I32P = C.POINTER(C.c_int32)
UINT64_MAX = (1 << 64) - 1


def _c(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _contig(p: Planes) -> Planes:
    return Planes(
        np.ascontiguousarray(p.x, np.uint64),
        np.ascontiguousarray(p.z, np.uint64),
        np.ascontiguousarray(p.flags, np.uint8),
        np.ascontiguousarray(p.val, np.float64),
    )


def _cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as fh:
            return "avx512f" in fh.read()
    except OSError:
        return False


class _Impl:
    prefix = ""

    def __init__(self, lib):
        self.lib = lib
        p = self.prefix
        f = lambda name: getattr(lib, p + name)  # noqa: E731
        self._new = f("sum_new")
        self._new.restype = C.c_void_p
        self._new.argtypes = [C.c_int, U64P, U64P, U8P, F64P, C.c_int64]
        self._free = f("sum_free")
        self._free.argtypes = [C.c_void_p]
        self._len = f("sum_len")
        self._len.restype = C.c_int64
        self._len.argtypes = [C.c_void_p]
        self._get = f("sum_get")
        self._get.argtypes = [C.c_void_p, U64P, U64P, U8P, F64P]

    # -- handle plumbing ------------------------------------------------
    def _make(self, p: Planes):
        p = _contig(p)
        h = self._new(p.array_size, _c(p.x, U64P), _c(p.z, U64P), _c(p.flags, U8P),
                      _c(p.val, F64P), p.n)
        if not h:
            raise ValueError(f"unsupported array size {p.array_size}")
        return h

    def _take(self, h, array_size: int) -> Planes:
        n = self._len(h)
        out = Planes.empty(array_size, n)
        self._get(h, _c(out.x, U64P), _c(out.z, U64P), _c(out.flags, U8P), _c(out.val, F64P))
        self._free(h)
        return out

    def _inplace(self, p: Planes, fn, *args) -> Planes:
        h = self._make(p)
        fn(h, *args)
        return self._take(h, p.array_size)

    def _scalar(self, p, fn, *args):
        h = self._make(p)
        try:
            return fn(h, *args)
        finally:
            self._free(h)

    def frobenius_norm2(self, p) -> float:
        return self._scalar(p, getattr(self.lib, self.prefix + "frobenius_norm2"))

    def lookup(self, p, x, z, f) -> float:
        x = np.ascontiguousarray(x, np.uint64)
        z = np.ascontiguousarray(z, np.uint64)
        return self._scalar(p, getattr(self.lib, self.prefix + "lookup"), _c(x, U64P),
                            _c(z, U64P), int(f))

    def apply_clifford(self, p, gate: int, c: int, t: int = 0):
        """Bulk Clifford gate number `gate` (the library's PL_GATE_* values)."""
        return self._inplace(p, getattr(self.lib, self.prefix + "apply_clifford"), int(gate),
                             int(c), int(t))

    def apply_rgate(self, p, axis: int, c: int, angle: float):
        """apply_RX / RY / RZ (axis 1 / 2 / 3)."""
        return self._inplace(p, getattr(self.lib, self.prefix + "apply_rgate"), int(axis),
                             int(c), float(angle))


class Oracle(_Impl):
    """The C restatement (oracle/paulib_oracle.c)."""

    prefix = "or_"

    def __init__(self):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        super().__init__(C.CDLL(path))
        L = self.lib
        for name in ("or_canonicalize", "or_sort_and_combine"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.or_cutoff.argtypes = [C.c_void_p, C.c_double]
        L.or_truncate_weight.argtypes = [C.c_void_p, C.c_uint64]
        L.or_trim.argtypes = [C.c_void_p, C.c_uint64]
        L.or_trim_protected.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
        L.or_apply_clifford.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint64]
        L.or_apply_rgate.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_double]
        for name, args in (("or_basis_state_expectation", [C.c_void_p, U64P]),
                           ("or_trace", [C.c_void_p, C.c_int]),
                           ("or_frobenius_norm2", [C.c_void_p]),
                           ("or_lookup", [C.c_void_p, U64P, U64P, C.c_uint8]),
                           ("or_trace_product", [C.c_void_p, C.c_void_p, C.c_int])):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = args
        L.or_apply_cnot.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]
        L.or_zero_state_expectation.restype = C.c_double
        L.or_zero_state_expectation.argtypes = [C.c_void_p]
        L.or_evolve.argtypes = [C.c_void_p, C.c_void_p]
        L.or_multiply.restype = C.c_void_p
        L.or_multiply.argtypes = [C.c_void_p, C.c_void_p]
        L.or_commutator.restype = C.c_void_p
        L.or_commutator.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.or_propagate.argtypes = [C.c_void_p, C.c_void_p, I32P, C.c_int64, C.c_void_p]

    def canonicalize(self, p):
        return self._inplace(p, self.lib.or_canonicalize)

    def sort_and_combine(self, p):
        return self._inplace(p, self.lib.or_sort_and_combine)

    def cutoff(self, p, eps):
        return self._inplace(p, self.lib.or_cutoff, float(eps))

    def truncate_weight(self, p, w):
        return self._inplace(p, self.lib.or_truncate_weight, int(w))

    def trim(self, p, m):
        return self._inplace(p, self.lib.or_trim, int(m))

    def basis_state_expectation(self, p, bit_words) -> float:
        w = np.ascontiguousarray(bit_words, np.uint64)
        return self._scalar(p, self.lib.or_basis_state_expectation, _c(w, U64P))

    def trace(self, p, num_qubits: int) -> float:
        return self._scalar(p, self.lib.or_trace, int(num_qubits))

    def trace_product(self, a, b, num_qubits: int) -> float:
        hb = self._make(b)
        try:
            return self._scalar(a, self.lib.or_trace_product, hb, int(num_qubits))
        finally:
            self._free(hb)

    def trim_protected(self, p, m, keep):
        hk = self._make(keep)
        try:
            return self._inplace(p, self.lib.or_trim_protected, int(m), hk)
        finally:
            self._free(hk)

    def apply_cnot(self, p, c, t):
        return self._inplace(p, self.lib.or_apply_cnot, int(c), int(t))

    def zero_state_expectation(self, p) -> float:
        h = self._make(p)
        r = self.lib.or_zero_state_expectation(h)
        self._free(h)
        return float(r)

    def multiply(self, a, b):
        ha, hb = self._make(a), self._make(b)
        h = self.lib.or_multiply(ha, hb)
        self._free(ha), self._free(hb)
        return self._take(h, a.array_size)

    def commutator(self, a, b, mul_i=False):
        ha, hb = self._make(a), self._make(b)
        h = self.lib.or_commutator(ha, hb, int(bool(mul_i)))
        self._free(ha), self._free(hb)
        return self._take(h, a.array_size)

    def evolve(self, p, rot):
        h, hr = self._make(p), self._make(rot)
        self.lib.or_evolve(h, hr)
        self._free(hr)
        return self._take(h, p.array_size)

    def propagate(self, p, rot, ops=None, max_weight=None, cutoff=0.0, max_terms=None):
        class Trunc(C.Structure):
            _fields_ = [("max_weight", C.c_uint64), ("cutoff", C.c_double),
                        ("max_terms", C.c_uint64)]

        t = Trunc(UINT64_MAX if max_weight is None else int(max_weight), float(cutoff),
                  UINT64_MAX if max_terms is None else int(max_terms))
        h, hr = self._make(p), self._make(rot)
        if ops is None:
            self.lib.or_propagate(h, hr, None, 0, C.byref(t))
        else:
            o = np.ascontiguousarray(ops, np.int32).reshape(-1, 3)
            self.lib.or_propagate(h, hr, _c(o, I32P), o.shape[0], C.byref(t))
        self._free(hr)
        return self._take(h, p.array_size)


class Reference(_Impl):
    """The reference's own implementation, compiled into oracle/_ref/."""

    prefix = "ref_"
    SUPPORTED_AS = (1, 2, 3, 4, 8, 16)

    def __init__(self, threads: int | None = None):
        names = ["libpaulib_ref.so", "libpaulib_ref_x86v3.so"]
        if platform.machine() == "x86_64" and not _cpu_has_avx512():
            names = names[::-1]
        path = None
        for nm in names:
            cand = os.path.join(HERE, "_ref", nm)
            if os.path.exists(cand):
                path = cand
                break
        if path is None:
            raise FileNotFoundError("oracle/_ref/libpaulib_ref*.so missing: run `make -C oracle`")
        self.path = path
        super().__init__(C.CDLL(path))
        L = self.lib
        for name in ("ref_canonicalize", "ref_sort_and_combine"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.ref_cutoff.argtypes = [C.c_void_p, C.c_double]
        L.ref_truncate_weight.argtypes = [C.c_void_p, C.c_uint64]
        L.ref_trim.argtypes = [C.c_void_p, C.c_uint64]
        L.ref_trim_protected.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
        L.ref_apply_clifford.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_uint64]
        L.ref_apply_rgate.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_double]
        for name, args in (("ref_basis_state_expectation", [C.c_void_p, C.c_char_p]),
                           ("ref_trace", [C.c_void_p]),
                           ("ref_frobenius_norm2", [C.c_void_p]),
                           ("ref_lookup", [C.c_void_p, U64P, U64P, C.c_uint8]),
                           ("ref_trace_product", [C.c_void_p, C.c_void_p])):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = args
        L.ref_apply_cnot.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]
        L.ref_zero_state_expectation.restype = C.c_double
        L.ref_zero_state_expectation.argtypes = [C.c_void_p]
        L.ref_evolve.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_multiply.restype = C.c_void_p
        L.ref_multiply.argtypes = [C.c_void_p, C.c_void_p]
        L.ref_commutator.restype = C.c_void_p
        L.ref_commutator.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.ref_propagate.argtypes = [C.c_void_p, C.c_void_p, I32P, C.c_int64, C.c_uint64,
                                    C.c_double, C.c_uint64]
        L.ref_max_threads.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        if threads is not None:
            L.ref_set_threads(int(threads))

    @property
    def threads(self) -> int:
        return int(self.lib.ref_max_threads())

    def set_threads(self, n: int):
        self.lib.ref_set_threads(int(n))

    def canonicalize(self, p):
        return self._inplace(p, self.lib.ref_canonicalize)

    def sort_and_combine(self, p):
        return self._inplace(p, self.lib.ref_sort_and_combine)

    def cutoff(self, p, eps):
        return self._inplace(p, self.lib.ref_cutoff, float(eps))

    def truncate_weight(self, p, w):
        return self._inplace(p, self.lib.ref_truncate_weight, int(w))

    def trim(self, p, m):
        return self._inplace(p, self.lib.ref_trim, int(m))

    # the reference build's sums have num_qubits = 64 * array_size
    def basis_state_expectation(self, p, bit_words) -> float:
        nq = 64 * p.array_size
        bits = "".join("1" if (int(bit_words[q // 64]) >> (q % 64)) & 1 else "0"
                       for q in range(nq))
        return self._scalar(p, self.lib.ref_basis_state_expectation, bits.encode())

    def trace(self, p, num_qubits: int) -> float:
        assert num_qubits == 64 * p.array_size
        return self._scalar(p, self.lib.ref_trace)

    def trace_product(self, a, b, num_qubits: int) -> float:
        assert num_qubits == 64 * a.array_size
        hb = self._make(b)
        try:
            return self._scalar(a, self.lib.ref_trace_product, hb)
        finally:
            self._free(hb)

    def trim_protected(self, p, m, keep):
        hk = self._make(keep)
        try:
            return self._inplace(p, self.lib.ref_trim_protected, int(m), hk)
        finally:
            self._free(hk)

    def apply_cnot(self, p, c, t):
        return self._inplace(p, self.lib.ref_apply_cnot, int(c), int(t))

    def zero_state_expectation(self, p) -> float:
        h = self._make(p)
        r = self.lib.ref_zero_state_expectation(h)
        self._free(h)
        return float(r)

    def multiply(self, a, b):
        ha, hb = self._make(a), self._make(b)
        h = self.lib.ref_multiply(ha, hb)
        self._free(ha), self._free(hb)
        return self._take(h, a.array_size)

    def commutator(self, a, b, mul_i=False):
        ha, hb = self._make(a), self._make(b)
        h = self.lib.ref_commutator(ha, hb, int(bool(mul_i)))
        self._free(ha), self._free(hb)
        return self._take(h, a.array_size)

    def evolve(self, p, rot):
        h, hr = self._make(p), self._make(rot)
        self.lib.ref_evolve(h, hr)
        self._free(hr)
        return self._take(h, p.array_size)

    def propagate(self, p, rot, ops=None, max_weight=None, cutoff=0.0, max_terms=None):
        h, hr = self._make(p), self._make(rot)
        mw = UINT64_MAX if max_weight is None else int(max_weight)
        mt = UINT64_MAX if max_terms is None else int(max_terms)
        if ops is None:
            self.lib.ref_propagate(h, hr, None, 0, mw, float(cutoff), mt)
        else:
            o = np.ascontiguousarray(ops, np.int32).reshape(-1, 3)
            self.lib.ref_propagate(h, hr, _c(o, I32P), o.shape[0], mw, float(cutoff), mt)
        self._free(hr)
        return self._take(h, p.array_size)

    def random_pauli_sum(self, array_size: int, terms: int, seed: int, num_qubits: int):
        """random_pauli_sum<64*array_size, double>(terms, seed, num_qubits)."""
        fn = self.lib.ref_random_pauli_sum
        fn.restype = C.c_void_p
        fn.argtypes = [C.c_int, C.c_int64, C.c_uint64, C.c_uint64]
        h = fn(int(array_size), int(terms), int(seed), int(num_qubits))
        if not h:
            raise ValueError(f"unsupported array size {array_size}")
        return self._take(h, array_size)

    # A handle-level multiply+canonicalize without the intermediate round trip,
    # used to time the reference's product+collate path.
    def multiply_canonicalize(self, a, b):
        ha, hb = self._make(a), self._make(b)
        h = self.lib.ref_multiply(ha, hb)
        self._free(ha), self._free(hb)
        self.lib.ref_canonicalize(h)
        return self._take(h, a.array_size)
