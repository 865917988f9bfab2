"""Reference-style scripts against the drop-in ``paulib`` package
(paulib_b200/python/paulib): the reference's factories and per-capacity
classes, run on the GPU, compared with the reference build and the oracle."""
import math
import os
import sys

import numpy as np
import pytest

from helpers import assert_keys_equal, assert_values_close, abs_scale
from paulib_b200.planes import Planes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "paulib_b200", "python"))

import paulib  # noqa: E402
from paulib import PauliString, PauliSum, TruncationOptions, _paulib  # noqa: E402

pytestmark = pytest.mark.gpu


def _planes(s) -> Planes:
    return Planes(*s.planes())


@pytest.mark.parametrize("nq", [20, 100])
def test_random_sums_product_and_commutator_vs_reference(cuda, reference, oracle, nq):
    aw = (nq + 63) // 64
    a = paulib.random_pauli_sum(nq, 300, seed=5)
    b = paulib.random_pauli_sum(nq, 200, seed=6)
    assert type(a).__name__ == f"PauliSum_{64 * aw}" and len(a) == 300
    A, B = reference.random_pauli_sum(aw, 300, 5, nq), reference.random_pauli_sum(aw, 200, 6, nq)
    assert_keys_equal(_planes(a), A)
    p = a * b
    p.canonicalize()
    raw = reference.multiply(A, B)
    want = reference.canonicalize(raw)
    assert_keys_equal(_planes(p), want)
    assert_values_close(_planes(p), want, abs_scale(oracle, raw))
    c = paulib.commutator(a, b)
    want_c = reference.canonicalize(reference.commutator(A, B))
    assert_keys_equal(_planes(c), want_c)
    assert_values_close(_planes(c), want_c, abs_scale(oracle, reference.commutator(A, B)))
    assert paulib.trace_product(a, b) == pytest.approx(
        reference.trace_product(A, B, 64 * aw), abs=1e-9)


def test_propagate_expectation_with_options(cuda, oracle):
    obs = PauliSum([("ZIIIII", 1.0), ("IIZIII", 0.5), ("IIIIXZ", 0.25)])
    rot = PauliSum([("XIIIII", 0.3), ("ZZIIII", 1.1), ("IXYIII", -0.7), ("IIIZZI", 0.4),
                    ("YIIIIX", 2.0), ("IIZXII", math.pi / 2)])
    opts = TruncationOptions()
    opts.max_weight = 4
    opts.coefficient_cutoff = 1e-3
    got = paulib.propagate_expectation(obs, rot, opts)
    o = oracle.propagate(_planes(obs), _planes(rot), None, max_weight=4, cutoff=1e-3)
    assert abs(got - oracle.zero_state_expectation(o)) <= 1e-10
    assert abs(paulib.propagate_expectation(obs, rot) -
               oracle.zero_state_expectation(oracle.propagate(_planes(obs), _planes(rot)))) <= 1e-10


def test_sum_methods_and_operators(cuda):
    s = PauliSum([("XYZ", 0.5), ("ZZI", 1.5), ("XYZ", 0.25)])
    assert type(s) is _paulib.PauliSum_64 and s.num_qubits() == 3
    s.push_back(PauliString("IXI"), 2.0)
    assert len(s) == 4 and s[3] == ("IXI", 2.0)
    s.set_X(1, 2)
    assert s[1][0] == "ZZX"
    assert s.term_weight(1) == 3 and s.term_weight(3) == 1
    ps = s.get_pauli_string(0)
    assert type(ps) is _paulib.PauliString_64 and str(ps) == "XYZ"
    assert s.commute(0, 2) and not s.commute(0, PauliString("ZII"))
    assert s.commute_with_Z(3, 0) and not s.commute_with_Z(3, 1)
    s.multiply_iZ(3, 1)  # iZ * X on qubit 1 = i (iY) = -Y
    assert s[3][0] == "-IYI"
    s.collate()  # sorted by (x, z, flags): x = 2 (IYI), 3 (XYZ), 4 (ZZX)
    assert str(s) == "2.000000 * -IYI\n0.750000 * XYZ\n1.500000 * ZZX\n"
    t = 2.0 * s
    assert [t[i][1] for i in range(len(t))] == [4.0, 1.5, 3.0]
    u = s * 3.0
    u -= s
    u.canonicalize()  # the sign of -IYI folds into its coefficient
    assert str(u) == "-4.000000 * IYI\n1.500000 * XYZ\n3.000000 * ZZX\n"
    z = s - s
    z.canonicalize()
    assert len(z) == 0
    n = -s
    assert [n[i][1] for i in range(len(n))] == [-2.0, -0.75, -1.5]
    with pytest.raises(IndexError):
        s.get_pauli_string(7)
    with pytest.raises(ValueError):
        s * PauliSum([("XX", 1.0)])
    e = _paulib.PauliSum_128(70)
    assert e.num_qubits() == 70 and len(e) == 0
    with pytest.raises(ValueError):
        _paulib.PauliSum_64(65)
