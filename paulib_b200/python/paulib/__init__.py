"""paulib -- the reference's Python package (python/paulib/__init__.py:1-173)
as a drop-in over this library: the same factories, names and exception
types, with every Pauli-sum method running on the GPU.

With ``paulib_b200/python`` on ``sys.path`` (or ``PYTHONPATH``), reference
scripts run unchanged::

    from paulib import PauliString, PauliSum, random_pauli_sum
    soa = PauliSum([("XYZZ", 0.5), ("ZZZY", 1.2)])
    soa.canonicalize()
"""
from __future__ import annotations

from typing import List, Sequence, Tuple, Union

from . import _paulib

SUPPORTED_CAPACITIES: List[int] = sorted(_paulib.SUPPORTED_CAPACITIES)
MAX_QUBITS: int = SUPPORTED_CAPACITIES[-1]


def _count_qubits(s: str) -> int:
    i = 0
    if i < len(s) and s[i] in "+-":
        i += 1
    if i < len(s) and s[i] == "i":
        i += 1
    return len(s) - i


def _capacity_for(n: int) -> int:
    if n < 1:
        raise ValueError("Qubit count must be at least 1.")
    for cap in SUPPORTED_CAPACITIES:
        if n <= cap:
            return cap
    raise ValueError(f"Qubit count {n} exceeds the maximum of {MAX_QUBITS} qubits.")


def _cls(prefix: str, cap: int):
    return getattr(_paulib, f"{prefix}_{cap}")


def PauliString(s: str):
    """A PauliString from ``[+|-][i]<pauli_chars>`` (X, Y, Z, I)."""
    return _cls("PauliString", _capacity_for(_count_qubits(s)))(s)


def PauliSum(terms: Union[str, Sequence[str], Sequence[Tuple[str, float]]],
             coefficient: float = 1.0):
    """A PauliSum with double coefficients from one string, a list of
    strings (coefficients 1.0) or a list of (string, coefficient) pairs."""
    if isinstance(terms, str):
        return _cls("PauliSum", _capacity_for(_count_qubits(terms)))([(terms, coefficient)])
    terms = list(terms)
    if not terms:
        raise ValueError("Cannot infer qubit count from an empty list. "
                         "Use a non-empty list or pass a single string.")
    strs = [t if isinstance(t, str) else t[0] for t in terms]
    return _cls("PauliSum", _capacity_for(max(_count_qubits(s) for s in strs)))(terms)


def random_pauli_sum(n_qubits: int, num_terms: int, seed: int = 42):
    """A random PauliSum with n_qubits qubits (the reference's draws)."""
    return getattr(_paulib, f"random_pauli_sum_{_capacity_for(n_qubits)}")(num_terms, seed,
                                                                          n_qubits)


TruncationOptions = _paulib.TruncationOptions


def _fn(name: str, obj):
    return getattr(_paulib, f"{name}_{type(obj).CAPACITY}")


def trace_product(a, b) -> float:
    """Re tr(A*B), computed without forming the product."""
    return _fn("trace_product", a)(a, b)


def commutator(a, b):
    """[A, B], canonicalized."""
    return _fn("commutator", a)(a, b)


def i_commutator(a, b):
    """i[A, B], canonicalized (Hermitian for Hermitian inputs)."""
    return _fn("i_commutator", a)(a, b)


def propagate_expectation(observable, rotations, options=None) -> float:
    """Pauli propagation: <0|U^dagger O U|0> for the rotation circuit U."""
    return _fn("propagate_expectation", observable)(observable, rotations, options)


__all__ = ["SUPPORTED_CAPACITIES", "MAX_QUBITS", "PauliString", "PauliSum", "random_pauli_sum",
           "TruncationOptions", "trace_product", "commutator", "i_commutator",
           "propagate_expectation", "_paulib"]
