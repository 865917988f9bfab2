"""The reference's Python surface (python/paulib/__init__.py:64-159 and the
PauliSum_<N> bindings, python/bindings.cpp:138-298) for the hot path, on
device-resident sums.

    from paulib_b200.paulib import PauliSum, TruncationOptions, commutator
    soa = PauliSum([("XYZZ", 0.5), ("ZZZY", 1.2)])
    soa.canonicalize()

Same names, argument meanings and exception types (ValueError for bad
input, IndexError for a bad term index).  Every method runs on the GPU
through the C ABI; there is no CPU path.
"""
from __future__ import annotations

from typing import Sequence, Tuple, Union

import numpy as np

from . import _abi
from . import strings
from .propagation import State

MAX_QUBITS = 64 * 16


class TruncationOptions:
    """TruncationOptions<double> (PauliPropagation.h:27-31)."""

    def __init__(self, max_weight=None, coefficient_cutoff=0.0, max_terms=None):
        self.max_weight = max_weight
        self.coefficient_cutoff = coefficient_cutoff
        self.max_terms = max_terms


def _capacity_words(n: int) -> int:
    if n < 1:
        raise ValueError("Qubit count must be at least 1.")
    if n > MAX_QUBITS:
        raise ValueError(f"Qubit count {n} exceeds the maximum of {MAX_QUBITS} qubits.")
    return (n + 63) // 64


def _count_qubits(s: str) -> int:
    i = 0
    if i < len(s) and s[i] in "+-":
        i += 1
    if i < len(s) and s[i] == "i":
        i += 1
    return len(s) - i


def _checked(fn, *args):
    try:
        return fn(*args)
    except _abi.PLError as e:
        if e.status == _abi.PL_ERR_INVALID_ARG:
            raise ValueError(str(e)) from None
        raise


class PauliString:
    """PauliString<N> (PauliStringCore.h:17-35): one string of x / z words and
    a flags byte (bit0 imaginary, bit1 sign), as a host value.  Its algebra
    (product, commutation) is O(words) bit arithmetic on the host, like the
    reference's stack object; sums of strings live and compute on the GPU.

        PauliString("XYZZ"), PauliString("+iXYZZ"), PauliString("-iXY")
    """

    CAPACITY = None  # qubits; set by the per-capacity classes

    def __init__(self, s: str = ""):
        words = None if self.CAPACITY is None else self.CAPACITY // 64
        if s == "":
            self._nq = 0
            aw = words or 1
            self.x, self.z, self.flags = [0] * aw, [0] * aw, 0
            return
        x, z, f, nq = strings.parse(s, words)
        self.x, self.z, self.flags, self._nq = list(x), list(z), int(f), int(nq)

    @classmethod
    def _of(cls, x, z, flags, nq):
        ps = cls.__new__(cls)
        ps.x, ps.z, ps.flags, ps._nq = [int(v) for v in x], [int(v) for v in z], int(flags), nq
        return ps

    def num_qubits(self) -> int:
        return self._nq

    def _same(self, other):
        if not isinstance(other, PauliString):
            raise TypeError("expected a PauliString")
        if other._nq != self._nq:
            raise ValueError(f"qubit count mismatch: {self._nq} vs {other._nq}")

    def _q(self, q):
        if not 0 <= q < self._nq:
            raise IndexError(f"qubit index {q} out of range for {self._nq} qubits")

    def inner_product(self, other) -> int:
        self._same(other)
        return strings.anticommute_words(self.x, self.z, other.x, other.z)

    def commute(self, other) -> bool:
        return self.inner_product(other) == 0

    def anti_commute(self, other) -> bool:
        return self.inner_product(other) == 1

    def multiply(self, other):
        """self := self * other."""
        self._same(other)
        self.x, self.z, self.flags = strings.multiply_words(self.x, self.z, self.flags,
                                                            other.x, other.z, other.flags)

    def __mul__(self, other):
        out = type(self)._of(self.x, self.z, self.flags, self._nq)
        out.multiply(other)
        return out

    def __imul__(self, other):
        self.multiply(other)
        return self

    def get_sign(self) -> bool:
        return bool(self.flags & 2)

    def get_phase(self) -> bool:
        return bool(self.flags & 1)

    def set_sign(self, v: bool):
        self.flags = (self.flags & 1) | (2 if v else 0)

    def set_phase(self, v: bool):
        self.flags = (self.flags & 2) | (1 if v else 0)

    def set_pauli(self, qubit: int, p: str):
        """Set qubit to 'X', 'Y', 'Z' or 'I'."""
        self._q(qubit)
        if p not in ("I", "X", "Y", "Z"):
            raise ValueError("Invalid Pauli character")
        w, b = divmod(qubit, 64)
        bit = 1 << b
        self.x[w] = (self.x[w] & ~bit) | (bit if p in "XY" else 0)
        self.z[w] = (self.z[w] & ~bit) | (bit if p in "YZ" else 0)

    def _single(self, axis: str, qubit: int) -> bool:
        self._q(qubit)
        w, b = divmod(qubit, 64)
        xb, zb = (self.x[w] >> b) & 1, (self.z[w] >> b) & 1
        return {"X": zb == 0, "Z": xb == 0, "Y": xb == zb}[axis]

    def commute_with_X(self, qubit: int) -> bool:
        return self._single("X", qubit)

    def commute_with_Z(self, qubit: int) -> bool:
        return self._single("Z", qubit)

    def commute_with_Y(self, qubit: int) -> bool:
        return self._single("Y", qubit)

    def _mul_site(self, p: str, qubit: int, imag: bool):
        self._q(qubit)
        one = PauliString._of([0] * len(self.x), [0] * len(self.z), 1 if imag else 0, self._nq)
        one.set_pauli(qubit, p)
        self.x, self.z, self.flags = strings.multiply_words(one.x, one.z, one.flags,
                                                            self.x, self.z, self.flags)

    def multiply_iX(self, qubit: int):
        self._mul_site("X", qubit, True)

    def multiply_iY(self, qubit: int):
        self._mul_site("Y", qubit, True)

    def multiply_iZ(self, qubit: int):
        self._mul_site("Z", qubit, True)

    def to_string(self) -> str:
        return strings.fmt(self.x, self.z, self.flags, self._nq)

    __str__ = to_string

    def __repr__(self) -> str:
        return f'PauliString("{self.to_string()}")'

    def __eq__(self, other) -> bool:
        return (isinstance(other, PauliString) and self._nq == other._nq and
                self.x == other.x and self.z == other.z and self.flags == other.flags)


class _PauliSum:
    """A Pauli sum with FP64 coefficients kept in device memory."""

    def __init__(self, num_qubits: int, x=None, z=None, f=None, v=None, state=None, words=None):
        self._nq = int(num_qubits)
        self._aw = int(words) if words is not None else _capacity_words(self._nq)
        self._st = state if state is not None else State(self._aw)
        if v is not None:
            self._st.upload(x, z, f, v)

    # -- accessors -------------------------------------------------------
    def num_qubits(self) -> int:
        return self._nq

    def __len__(self) -> int:
        return self._st.size()

    @property
    def coefficients(self):
        return list(self._st.download()[3])

    def planes(self):
        """(x (AS, n), z (AS, n), flags, values) copied to the host."""
        return self._st.download()

    def get_str(self) -> str:
        x, z, f, v = self._st.download()
        return strings.get_str(x, z, f, v, self._nq)

    __str__ = get_str
    __repr__ = get_str

    def __getitem__(self, i: int):
        x, z, f, v = self._st.download()
        if not 0 <= i < v.shape[0]:
            raise IndexError("term index out of range")
        return strings.fmt(x[:, i], z[:, i], f[i], self._nq), float(v[i])

    def _check_same(self, other):
        if not isinstance(other, _PauliSum):
            raise TypeError("expected a PauliSum")
        if other._nq != self._nq:
            raise ValueError("Pauli sums have different qubit counts")

    def _empty_like(self) -> "_PauliSum":
        out = type(self).__new__(type(self))
        _PauliSum.__init__(out, self._nq, words=self._aw)
        return out

    def _copy(self) -> "_PauliSum":
        out = self._empty_like()
        _checked(out._st._lib.pl_state_append, out._st._h, self._st._h)
        return out

    def _term(self, i: int):
        n = len(self)
        if not 0 <= i < n:
            raise IndexError(f"term index {i} out of range for {n} terms")

    def _edit(self, i: int, fn):
        """Per-term edit (the reference's public SoA fields): host copy of the
        planes, fn(x, z, f, v) edits term i in place, upload back."""
        self._term(i)
        x, z, f, v = self._st.download()
        fn(x, z, f, v)
        self._st.upload(x, z, f, v)

    def _string_cls(self):
        return PauliString

    # -- data model (PauliSumCore.h) ---------------------------------------
    def reserve(self, capacity: int):
        """Capacity hint; device buffers grow on demand."""

    def push_back(self, pauli_string: PauliString, coefficient: float = 1.0):
        if pauli_string.num_qubits() > self._nq:
            raise ValueError("Pauli string has more qubits than the sum")
        one = self._empty_like()
        one._st.upload(np.array(pauli_string.x[: self._aw] + [0] * (self._aw - len(pauli_string.x)),
                                np.uint64).reshape(self._aw, 1),
                       np.array(pauli_string.z[: self._aw] + [0] * (self._aw - len(pauli_string.z)),
                                np.uint64).reshape(self._aw, 1),
                       np.array([pauli_string.flags], np.uint8), np.array([coefficient], np.float64))
        _checked(self._st._lib.pl_state_append, self._st._h, one._st._h)

    def get_pauli_string(self, i: int) -> PauliString:
        x, z, f, v = self._st.download()
        if not 0 <= i < v.shape[0]:
            raise IndexError(f"term index {i} out of range for {v.shape[0]} terms")
        return self._string_cls()._of(x[:, i], z[:, i], f[i], self._nq)

    def term_weight(self, i: int) -> int:
        ps = self.get_pauli_string(i)
        return sum(bin(a | b).count("1") for a, b in zip(ps.x, ps.z))

    def commute(self, i: int, other) -> bool:
        """Whether term i commutes with a PauliString, or with term j."""
        a = self.get_pauli_string(i)
        b = self.get_pauli_string(other) if isinstance(other, int) else other
        return a.commute(b)

    def commute_with_X(self, i: int, qubit: int) -> bool:
        return self.get_pauli_string(i).commute_with_X(qubit)

    def commute_with_Z(self, i: int, qubit: int) -> bool:
        return self.get_pauli_string(i).commute_with_Z(qubit)

    def commute_with_Y(self, i: int, qubit: int) -> bool:
        return self.get_pauli_string(i).commute_with_Y(qubit)

    def _set_site(self, i: int, qubit: int, p: str):
        if not 0 <= qubit < self._nq:
            raise IndexError(f"qubit index {qubit} out of range for {self._nq} qubits")
        w, b = divmod(qubit, 64)
        bit = np.uint64(1) << np.uint64(b)

        def fn(x, z, f, v):
            x[w, i] = (x[w, i] & ~bit) | (bit if p in "XY" else np.uint64(0))
            z[w, i] = (z[w, i] & ~bit) | (bit if p in "YZ" else np.uint64(0))
        self._edit(i, fn)

    def set_X(self, i: int, qubit: int):
        self._set_site(i, qubit, "X")

    def set_Y(self, i: int, qubit: int):
        self._set_site(i, qubit, "Y")

    def set_Z(self, i: int, qubit: int):
        self._set_site(i, qubit, "Z")

    def _left_multiply(self, i: int, ps: PauliString):
        def fn(x, z, f, v):
            nx, nz, nf = strings.multiply_words(ps.x, ps.z, ps.flags, x[:, i], z[:, i], f[i])
            x[:, i] = nx
            z[:, i] = nz
            f[i] = nf
        self._edit(i, fn)

    def multiply_at(self, i: int, pauli_string: PauliString):
        """Left-multiply term i by a PauliString (PauliSumOperations.h:186-209)."""
        if pauli_string.num_qubits() != self._nq:
            raise ValueError("qubit count mismatch")
        self._left_multiply(i, pauli_string)

    def _mul_site(self, i, p, qubit):
        if not 0 <= qubit < self._nq:
            raise IndexError(f"qubit index {qubit} out of range for {self._nq} qubits")
        one = PauliString._of([0] * self._aw, [0] * self._aw, 1, self._nq)
        one.set_pauli(qubit, p)
        self._left_multiply(i, one)

    def multiply_iX(self, i: int, qubit: int):
        self._mul_site(i, "X", qubit)

    def multiply_iY(self, i: int, qubit: int):
        self._mul_site(i, "Y", qubit)

    def multiply_iZ(self, i: int, qubit: int):
        self._mul_site(i, "Z", qubit)

    def scale(self, c: float):
        """Every coefficient times c (PauliSumCore.h: value *= c), on the
        device: the product with the identity string of coefficient c."""
        ident = self._empty_like()
        ident._st.upload(np.zeros((self._aw, 1), np.uint64), np.zeros((self._aw, 1), np.uint64),
                         np.zeros(1, np.uint8), np.array([float(c)]))
        _checked(_abi.check, self._st._lib.pl_state_multiply(self._st._h, ident._st._h),
                 "pl_state_multiply")

    # -- hot-path methods (reference names) ------------------------------
    def collate(self):
        """sort_and_combine (PauliSumOperations.h:369-461)."""
        self._st.sort_and_combine()

    def canonicalize(self):
        self._st.canonicalize()

    def cutoff(self, eps: float):
        self._st.cutoff(eps)

    def truncate_weight(self, max_weight: int):
        self._st.truncate_weight(max_weight)

    def trim(self, max_terms: int, keep: "_PauliSum | None" = None):
        if keep is not None:
            self._check_same(keep)
        self._st.trim(max_terms, None if keep is None else keep._st)

    def multiply(self, rhs: "_PauliSum"):
        """self := self * rhs (polynomial product, PauliSumOperations.h:256-306)."""
        self._check_same(rhs)
        _checked(_abi.check, self._st._lib.pl_state_multiply(self._st._h, rhs._st._h),
                 "pl_state_multiply")

    def evolve(self, rotations: "_PauliSum"):
        """Apply the rotations (generator = term, angle = coefficient) in order."""
        self._check_same(rotations)
        x, z, f, v = rotations._st.download()
        self._st.evolve(x, z, f, v)

    def apply_CNOT(self, control: int, target: int):
        if not (0 <= control < self._nq and 0 <= target < self._nq):
            raise IndexError("qubit index out of range")
        _checked(self._st.apply_cnot, control, target)

    def zero_state_expectation(self) -> float:
        return self._st.zero_state_expectation()

    # -- reductions (PauliSumUtils.h:178-268, 400-410) ---------------------
    def basis_state_expectation(self, bits: str) -> float:
        if len(bits) != self._nq:
            raise ValueError(f"basis_state_expectation: bit string length {len(bits)} does "
                             f"not match {self._nq} qubits")
        if any(c not in "01" for c in bits):
            raise ValueError("basis_state_expectation: bit string must contain only '0'/'1'")
        w = np.zeros(self._aw, np.uint64)
        for q, c in enumerate(bits):
            if c == "1":
                w[q // 64] |= np.uint64(1) << np.uint64(q % 64)
        return self._st.basis_state_expectation(w)

    def trace(self) -> float:
        return self._st.trace(self._nq)

    def frobenius_norm2(self) -> float:
        return self._st.frobenius_norm2()

    def lookup(self, pauli_string: str) -> float:
        x, z, f, nq = strings.parse(pauli_string, self._aw)
        if nq > self._nq:
            raise ValueError("Pauli string has more qubits than the sum")
        return self._st.lookup(np.array(x, np.uint64), np.array(z, np.uint64), f)

    # -- Clifford and rotation gates (PauliSumClifford.h, PauliSumOperations.h:29-104)
    def _q(self, *qs):
        for q in qs:
            if not 0 <= q < self._nq:
                raise IndexError("qubit index out of range")

    def _g1(self, name, qubit):
        self._q(qubit)
        _checked(self._st.apply_clifford, name, qubit, 0)

    def _g2(self, name, a, b):
        self._q(a, b)
        if a == b:
            raise ValueError("two-qubit gate needs two different qubits")
        _checked(self._st.apply_clifford, name, a, b)

    def apply_H(self, qubit): self._g1("H", qubit)
    def apply_H_YZ(self, qubit): self._g1("H_YZ", qubit)
    def apply_H_XY(self, qubit): self._g1("H_XY", qubit)
    def apply_S(self, qubit): self._g1("S", qubit)
    def apply_SX(self, qubit): self._g1("SQRT_X", qubit)
    def apply_SY(self, qubit): self._g1("SQRT_Y", qubit)
    def apply_X(self, qubit): self._g1("X", qubit)
    def apply_Y(self, qubit): self._g1("Y", qubit)
    def apply_Z(self, qubit): self._g1("Z", qubit)
    def apply_I(self, qubit): self._g1("I", qubit)
    def apply_CZ(self, control, target): self._g2("CZ", control, target)
    def apply_CY(self, control, target): self._g2("CY", control, target)
    def apply_XC_X(self, control, target): self._g2("XC_X", control, target)
    def apply_XC_Y(self, control, target): self._g2("XC_Y", control, target)
    def apply_XC_Z(self, control, target): self._g2("XC_Z", control, target)
    def apply_YC_X(self, control, target): self._g2("YC_X", control, target)
    def apply_YC_Y(self, control, target): self._g2("YC_Y", control, target)
    def apply_YC_Z(self, control, target): self._g2("YC_Z", control, target)
    def apply_SWAP(self, qubit1, qubit2): self._g2("SWAP", qubit1, qubit2)
    def apply_iSWAP(self, qubit1, qubit2): self._g2("ISWAP", qubit1, qubit2)

    def apply_RX(self, qubit, angle):
        self._q(qubit)
        self._st.apply_rotation_gate("X", qubit, angle)

    def apply_RY(self, qubit, angle):
        self._q(qubit)
        self._st.apply_rotation_gate("Y", qubit, angle)

    def apply_RZ(self, qubit, angle):
        self._q(qubit)
        self._st.apply_rotation_gate("Z", qubit, angle)

    # -- operators ---------------------------------------------------------
    def __mul__(self, other):
        out = self._copy()
        if isinstance(other, (int, float)):
            out.scale(float(other))
        else:
            out.multiply(other)
        return out

    def __rmul__(self, other):
        if not isinstance(other, (int, float)):
            return NotImplemented
        out = self._copy()
        out.scale(float(other))
        return out

    def __imul__(self, other):
        if isinstance(other, (int, float)):
            self.scale(float(other))
        else:
            self.multiply(other)
        return self

    def __iadd__(self, other):
        """append, then sort_and_combine (PauliSumCore.h:210-237)."""
        self._check_same(other)
        _checked(_abi.check, self._st._lib.pl_state_append(self._st._h, other._st._h),
                 "pl_state_append")
        self._st.sort_and_combine()
        return self

    def __add__(self, other):
        out = self._copy()
        out += other
        return out

    def __isub__(self, other):
        """append -1 * other, then sort_and_combine (PauliSumCore.h:246-250)."""
        self._check_same(other)
        neg = other._copy()
        neg.scale(-1.0)
        return self.__iadd__(neg)

    def __sub__(self, other):
        out = self._copy()
        out -= other
        return out

    def __neg__(self):
        out = self._copy()
        out.scale(-1.0)
        return out


def PauliSum(terms: Union[str, Sequence[str], Sequence[Tuple[str, float]]],
             coefficient: float = 1.0):
    """A device-resident Pauli sum from strings, as the reference's factory."""
    if isinstance(terms, str):
        terms = [(terms, coefficient)]
    terms = list(terms)
    if not terms:
        raise ValueError("Cannot infer qubit count from an empty list. "
                         "Use a non-empty list or pass a single string.")
    nq = max(_count_qubits(t if isinstance(t, str) else t[0]) for t in terms)
    aw = _capacity_words(nq)
    try:
        x, z, f, v, _ = strings.planes_from_terms(terms, aw)
    except ValueError:
        raise
    return _PauliSum(nq, x, z, f, v)


def commutator(a: _PauliSum, b: _PauliSum) -> _PauliSum:
    """[A, B], canonicalized."""
    return _comm(a, b, 0)


def i_commutator(a: _PauliSum, b: _PauliSum) -> _PauliSum:
    """i[A, B], canonicalized (Hermitian for Hermitian inputs)."""
    return _comm(a, b, 1)


def _comm(a, b, mul_i):
    a._check_same(b)
    out = a._empty_like()
    _abi.check(out._st._lib.pl_state_commutator(out._st._h, a._st._h, b._st._h, mul_i),
               "pl_state_commutator")
    out.canonicalize()
    return out


def trace_product(a: _PauliSum, b: _PauliSum) -> float:
    """Re tr(A*B), computed without forming the product."""
    if a._nq != b._nq:
        raise ValueError("trace_product: qubit-count mismatch")
    return a._st.trace_product(b._st, a._nq)


def propagate_expectation(observable: _PauliSum, rotations: _PauliSum,
                          options: TruncationOptions | None = None) -> float:
    """Pauli propagation: <0|U^dagger O U|0> for the rotation circuit U
    (generator = term, angle = coefficient; PauliPropagation.h:65-71)."""
    observable._check_same(rotations)
    o = options or TruncationOptions()
    out = observable._copy()
    x, z, f, v = rotations._st.download()
    out._st.propagate(x, z, f, v, None, o.max_weight, o.coefficient_cutoff, o.max_terms)
    return out.zero_state_expectation()


__all__ = ["PauliString", "PauliSum", "TruncationOptions", "commutator", "i_commutator",
           "trace_product", "propagate_expectation", "MAX_QUBITS"]
