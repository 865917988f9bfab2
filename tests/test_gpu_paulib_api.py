"""The Python surface with the reference's names (paulib_b200.paulib) on the
GPU: known answers of the reference's tests and Python example, and the
reference's exception types."""
import math

import numpy as np
import pytest

from paulib_b200 import paulib as P

pytestmark = pytest.mark.gpu


def test_factories_and_printing(cuda):
    s = P.PauliSum([("XY", 2.0), ("ZZ", 1.0), ("XY", 3.0)])
    assert len(s) == 3 and s.num_qubits() == 2
    s.collate()
    assert str(s) == "1.000000 * ZZ\n5.000000 * XY\n"
    assert s[1] == ("XY", 5.0)
    with pytest.raises(IndexError):
        s[5]
    assert P.PauliSum("XYZ", 0.5).coefficients == [0.5]
    with pytest.raises(ValueError):
        P.PauliSum([])
    with pytest.raises(ValueError):
        P.PauliSum([("XQ", 1.0)])


def test_algebra(cuda):
    a, b = P.PauliSum([("X", 1.0)]), P.PauliSum([("Y", 1.0)])
    assert str(a * b) == "1.000000 * iZ\n"
    c = P.PauliSum([("XX", 1.0), ("ZZ", 2.0)])
    c += P.PauliSum([("XX", 3.0)])
    assert str(c) == "2.000000 * ZZ\n4.000000 * XX\n"
    # canonicalized, as the reference binding returns it (bindings.cpp:318-331):
    # the sign of -i Y folds into the coefficient
    comm = P.commutator(P.PauliSum([("X", 1.5)]), P.PauliSum([("Z", 2.0)]))
    assert str(comm) == "-6.000000 * iY\n"
    ic = P.i_commutator(P.PauliSum([("X", 1.5)]), P.PauliSum([("Z", 2.0)]))
    assert str(ic) == "6.000000 * Y\n"
    with pytest.raises(ValueError):
        a.multiply(P.PauliSum([("XX", 1.0)]))


def test_truncation_and_gates(cuda):
    s = P.PauliSum([("XI", 0.1), ("ZI", -5.0), ("IZ", 0.3), ("YI", 2.0)])
    s.trim(2)
    assert sorted(s.coefficients) == [-5.0, 2.0]
    s = P.PauliSum([("XII", 0.5), ("XYZ", 0.01), ("ZZI", -0.2)])
    s.cutoff(0.05)
    s.truncate_weight(1)
    assert str(s) == "0.500000 * XII\n"
    t = P.PauliSum([("XZ", 1.0)])
    t.apply_CNOT(0, 1)
    assert str(t) == "1.000000 * -YY\n"
    e = P.PauliSum([("X", 1.0)])
    e.evolve(P.PauliSum([("Z", math.pi / 3)]))
    assert e.coefficients == [math.cos(math.pi / 3), -math.sin(math.pi / 3)]
    z = P.PauliSum([("II", 1.5), ("ZI", 2.0), ("ZZ", 4.0), ("XI", 8.0), ("IY", 16.0)])
    assert z.zero_state_expectation() == 7.5


def test_propagate_expectation_matches_oracle(cuda, oracle):
    from helpers import planes
    obs = [("ZIIIII", 1.0), ("IIZIII", 0.5)]
    rot = [("XIIIII", 0.3), ("IYIIII", 1.1), ("ZXIIII", 0.7), ("IIXIII", 2.0), ("IIIZZX", 0.4)]
    opts = P.TruncationOptions(max_weight=3, coefficient_cutoff=1e-3)
    g = P.propagate_expectation(P.PauliSum(obs), P.PauliSum(rot), opts)
    o = oracle.propagate(planes(obs), planes(rot), None, max_weight=3, cutoff=1e-3)
    assert abs(g - oracle.zero_state_expectation(o)) <= 1e-10
