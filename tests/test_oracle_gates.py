"""Clifford and rotation gates: the C restatement and the reference build
against the reference's own known answers, and against each other on seeded
random sums (bit for bit)."""
import math

import pytest

from gates_golden import GATE, ONE_QUBIT, ROTATIONS, TWO_QUBIT
from helpers import assert_keys_equal, bit_identical, planes, random_sum, to_str


@pytest.fixture(params=["oracle", "reference"])
def impl(request, oracle):
    return oracle if request.param == "oracle" else request.getfixturevalue("reference")


@pytest.mark.parametrize("gate", sorted(ONE_QUBIT))
def test_one_qubit_truth_tables(impl, gate):
    for inp, out in ONE_QUBIT[gate].items():
        got = impl.apply_clifford(planes([(inp, 1.0)]), GATE[gate], 0)
        assert to_str(got, 1) == f"1.000000 * {out}\n", (gate, inp)


@pytest.mark.parametrize("gate", sorted(TWO_QUBIT))
def test_two_qubit_truth_tables(impl, gate):
    for inp, out in TWO_QUBIT[gate].items():
        got = impl.apply_clifford(planes([(inp, 1.0)]), GATE[gate], 0, 1)
        assert to_str(got, 2) == f"1.000000 * {out}\n", (gate, inp)


def test_iswap_is_swap_cz_s_s(impl):
    # CliffordExtendedTests.cpp:256-275
    for inp in ("II", "XI", "IY", "ZZ", "XY", "YZ"):
        a = impl.apply_clifford(planes([(inp, 1.0)]), GATE["ISWAP"], 0, 1)
        b = planes([(inp, 1.0)])
        for g, q in (("SWAP", (0, 1)), ("CZ", (0, 1)), ("S", (0,)), ("S", (1,))):
            b = impl.apply_clifford(b, GATE[g], *q)
        assert to_str(a, 2) == to_str(b, 2)
    assert to_str(impl.apply_clifford(planes([("XI", 1.0)]), GATE["ISWAP"], 0, 1), 2) == \
        "1.000000 * ZY\n"


def test_h_sequence_and_high_qubit(impl):
    # PauliSumTests.cpp:313-325, 390-395
    s = planes([("IZXY", 1.0)])
    for q, exp in ((0, "IZXY"), (1, "IXXY"), (2, "IXZY"), (3, "-IXZY")):
        s = impl.apply_clifford(s, GATE["H"], q)
        assert to_str(s, 4) == f"1.000000 * {exp}\n"
    s = impl.apply_clifford(planes([("IIIIIIIIXIIIIIII", 1.0)]), GATE["H"], 8)
    assert to_str(s, 16) == "1.000000 * IIIIIIIIZIIIIIII\n"


@pytest.mark.parametrize("case", range(len(ROTATIONS)))
def test_rotation_gates(impl, case):
    axis, inp, exp = ROTATIONS[case]
    got = impl.apply_rgate(planes(inp), axis, 0, math.pi / 3)
    assert to_str(got, 1) == exp


@pytest.mark.parametrize("words", [1, 2])
def test_gates_match_reference(oracle, reference, words):
    s = random_sum(400, words, 17 + words, None, "normal")
    nq = 64 * words
    for gate in range(1, 22):
        c, t = 5, nq - 3
        o = oracle.apply_clifford(s, gate, c, t)
        r = reference.apply_clifford(s, gate, c, t)
        assert_keys_equal(o, r)
        assert bit_identical(o, r)
    for axis in (1, 2, 3):
        o = oracle.apply_rgate(s, axis, 7, 0.37)
        r = reference.apply_rgate(s, axis, 7, 0.37)
        assert_keys_equal(o, r)
        assert abs(o.val - r.val).max() <= 1e-15 * abs(r.val).max()
