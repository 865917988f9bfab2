"""The reference's Python package names (python/paulib/__init__.py,
python/bindings.cpp:300-379) from paulib_b200/python/paulib, host side:
capacity dispatch, the PauliString value type against the oracle's
product and commutation, and random_pauli_sum's draws against the
reference build's own random_pauli_sum."""
import os
import sys

import numpy as np
import pytest

from helpers import planes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "paulib_b200", "python"))

import paulib  # noqa: E402
from paulib import PauliString, _paulib  # noqa: E402


def test_names_and_capacities():
    assert paulib.SUPPORTED_CAPACITIES == [64 * k for k in range(1, 17)]
    assert paulib.MAX_QUBITS == 1024
    for cap in paulib.SUPPORTED_CAPACITIES:
        for name in ("PauliString", "PauliSum", "random_pauli_sum", "commutator",
                     "i_commutator", "trace_product", "propagate_expectation"):
            assert hasattr(_paulib, f"{name}_{cap}")
    assert type(PauliString("XYZ")).__name__ == "PauliString_64"
    assert type(PauliString("X" * 65)).__name__ == "PauliString_128"
    with pytest.raises(ValueError):
        PauliString("X" * 1025)
    with pytest.raises(ValueError):
        PauliString("XQ")
    o = paulib.TruncationOptions()
    assert o.max_weight == (1 << 64) - 1 and o.coefficient_cutoff == 0.0


@pytest.mark.parametrize("a", ["X", "Y", "Z", "I", "iX", "-Y", "-iZ"])
@pytest.mark.parametrize("b", ["X", "Y", "Z", "I", "iY"])
def test_pauli_string_products_match_oracle(oracle, a, b):
    # PauliSumTests.cpp:65-199: the single-qubit Cayley table with phases
    pa, pb = PauliString(a), PauliString(b)
    got = pa * pb
    want = oracle.multiply(planes([(a, 1.0)]), planes([(b, 1.0)]))  # lhs * rhs
    assert got.x[0] == int(want.x[0, 0]) and got.z[0] == int(want.z[0, 0])
    assert got.flags == int(want.flags[0])
    assert pa.commute(pb) == (oracle.commutator(planes([(a, 1.0)]), planes([(b, 1.0)])).n == 0)


def test_pauli_string_accessors():
    p = PauliString("-iXYZI")
    assert p.num_qubits() == 4 and p.get_sign() and p.get_phase()
    p.set_sign(False)
    p.set_pauli(3, "Y")
    assert str(p) == "iXYZY"
    assert p.commute_with_Z(2) and not p.commute_with_X(2) and not p.commute_with_Y(0)
    p.multiply_iZ(0)  # iZ * X = i (iY) = -Y; times the existing i: -iY
    assert str(p) == "-iYYZY"
    with pytest.raises(IndexError):
        p.set_pauli(4, "X")
    assert PauliString("XY") == PauliString("XY") and PauliString("XY") != PauliString("YX")


@pytest.mark.parametrize("nq,terms,seed", [(20, 40, 42), (100, 25, 7), (256, 9, 123)])
def test_random_pauli_sum_draws_match_reference(reference, nq, terms, seed):
    from paulib_b200.strings import random_planes
    aw = (nq + 63) // 64
    r = reference.random_pauli_sum(aw, terms, seed, nq)
    x, z, f, v = random_planes(terms, seed, nq, aw)
    assert np.array_equal(r.x, x) and np.array_equal(r.z, z)
    assert np.array_equal(r.flags, f) and np.array_equal(r.val, v)


def test_mt19937_64_known_value():
    # the C++ standard's check value: the 10000th output of a
    # default-constructed std::mt19937_64
    from paulib_b200.strings import MT19937_64
    g = MT19937_64()
    for _ in range(9999):
        g()
    assert g() == 9981545732273789042
