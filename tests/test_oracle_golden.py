"""Pin the CPU oracle (and the reference build) to the reference's own
known-answer tests.

Each case restates an assertion of the reference's GoogleTest suite
(tests/PauliSumTests.cpp, tests/GpuPauliSumTests.cpp; file:line cited per
test) on the hot-path functions: Cayley table and phases, outer-product
order, sort_and_combine, canonicalize, cutoff / truncate_weight, CNOT truth
table, evolve fast paths, zero_state_expectation.  Both CPU implementations
must give the reference's expected answers.
"""
import math

import numpy as np
import pytest

from helpers import planes, random_sum, to_str
from paulib_b200.planes import Planes

IMPLS = ["oracle", "reference"]


@pytest.fixture(params=IMPLS)
def impl(request, oracle):
    if request.param == "oracle":
        return oracle
    return request.getfixturevalue("reference")


# PauliSumTests.cpp:397-414 -- single-qubit Cayley table with phases.
CAYLEY = {
    "I": {"I": "I", "X": "X", "Y": "Y", "Z": "Z"},
    "X": {"I": "X", "X": "I", "Y": "iZ", "Z": "-iY"},
    "Y": {"I": "Y", "X": "-iZ", "Y": "I", "Z": "iX"},
    "Z": {"I": "Z", "X": "iY", "Y": "-iX", "Z": "I"},
}


@pytest.mark.parametrize("row", "IXYZ")
@pytest.mark.parametrize("col", "IXYZ")
def test_cayley_table(impl, row, col):
    out = impl.multiply(planes([(row, 1.0)]), planes([(col, 1.0)]))
    assert to_str(out, 1) == f"1.000000 * {CAYLEY[row][col]}\n"


# PauliSumTests.cpp:110-143 -- flag encodings X*Y = iZ (0x01), Y*X = -iZ (0x03).
def test_phase_flags(impl):
    assert int(impl.multiply(planes([("X", 1.0)]), planes([("Y", 1.0)])).flags[0]) == 0x01
    assert int(impl.multiply(planes([("Y", 1.0)]), planes([("X", 1.0)])).flags[0]) == 0x03


# PauliSumTests.cpp:421-454 -- outer product equals per-pair scalar products
# in result[i*n + j] = lhs[j] * rhs[i] order (13x7 and the 2-word case).
@pytest.mark.parametrize("words,n,m", [(1, 13, 7), (2, 13, 7), (1, 3, 2)])
def test_outer_product_order(impl, oracle, words, n, m):
    lhs = random_sum(n, words, 42)
    rhs = random_sum(m, words, 99)
    out = impl.multiply(lhs, rhs)
    assert out.n == n * m
    for i in range(m):
        for j in range(n):
            one = oracle.multiply(
                Planes(lhs.x[:, j:j + 1], lhs.z[:, j:j + 1], lhs.flags[j:j + 1], lhs.val[j:j + 1]),
                Planes(rhs.x[:, i:i + 1], rhs.z[:, i:i + 1], rhs.flags[i:i + 1], rhs.val[i:i + 1]))
            t = i * n + j
            assert np.array_equal(out.x[:, t], one.x[:, 0])
            assert np.array_equal(out.z[:, t], one.z[:, 0])
            assert out.flags[t] == one.flags[0]
            assert out.val[t] == lhs.val[j] * rhs.val[i]


# PauliSumTests.cpp:456-462 -- an empty operand gives an empty product.
def test_empty_operand(impl):
    some = random_sum(5, 1, 1)
    empty = Planes.empty(1, 0)
    assert impl.multiply(some, empty).n == 0
    assert impl.multiply(empty, some).n == 0


# PauliSumTests.cpp:514-561 -- sort_and_combine behaviour.
def test_sort_and_combine_merges(impl):
    out = impl.sort_and_combine(planes([("XY", 2.0), ("ZZ", 1.0), ("XY", 3.0)]))
    assert to_str(out, 2) == "1.000000 * ZZ\n5.000000 * XY\n"


def test_sort_and_combine_sign_is_key(impl):
    out = impl.sort_and_combine(planes([("X", 2.0), ("-X", 3.0)]))
    assert to_str(out, 1) == "2.000000 * X\n3.000000 * -X\n"


def test_sort_and_combine_keeps_exact_zero(impl):
    out = impl.sort_and_combine(planes([("X", 2.0), ("X", -2.0)]))
    assert out.n == 1 and out.val[0] == 0.0


def test_sort_and_combine_empty_and_single(impl):
    assert impl.sort_and_combine(Planes.empty(1, 0)).n == 0
    assert to_str(impl.sort_and_combine(planes([("Y", 1.5)])), 1) == "1.500000 * Y\n"


def test_sort_and_combine_idempotent(impl):
    s = planes([("XY", 1.0), ("II", 4.0), ("XY", 1.0), ("ZZ", 2.0), ("II", -1.0)])
    once = impl.sort_and_combine(s)
    twice = impl.sort_and_combine(once)
    assert to_str(once, 2) == to_str(twice, 2)
    assert np.array_equal(once.val, twice.val)


# PauliSumTests.cpp:567-646 -- `+=` is append + sort_and_combine.
def test_add_is_append_then_combine(impl):
    a = planes([("XX", 1.0), ("ZZ", 2.0)])
    b = planes([("XX", 3.0)])
    cat = Planes(np.concatenate([a.x, b.x], 1), np.concatenate([a.z, b.z], 1),
                 np.concatenate([a.flags, b.flags]), np.concatenate([a.val, b.val]))
    assert to_str(impl.sort_and_combine(cat), 2) == "2.000000 * ZZ\n4.000000 * XX\n"


# PauliSumTests.cpp:689-712, 1029-1037 -- zero_state_expectation.
def test_zero_state_only_iz(impl):
    s = planes([("II", 1.5), ("ZI", 2.0), ("ZZ", 4.0), ("XI", 8.0), ("IY", 16.0)])
    assert impl.zero_state_expectation(s) == 7.5


def test_zero_state_sign_and_imaginary(impl):
    assert impl.zero_state_expectation(planes([("-Z", 3.0), ("Z", 1.0)])) == -2.0
    assert impl.zero_state_expectation(planes([("iZ", 3.0), ("-iZ", 5.0), ("I", 1.0)])) == 1.0
    assert impl.zero_state_expectation(Planes.empty(1, 0)) == 0.0


def test_zero_state_multiword_x(impl):
    with_x = ["I"] * 128
    with_x[100] = "X"
    s = planes([("".join(with_x), 5.0), ("Z" * 128, 2.0)])
    assert impl.zero_state_expectation(s) == 2.0


# PauliSumTests.cpp:826-879 -- CNOT truth table, high indices, cross word.
CNOT = {"II": "II", "IX": "IX", "IY": "ZY", "IZ": "ZZ", "XI": "XX", "XX": "XI",
        "XY": "YZ", "XZ": "-YY", "YI": "YX", "YX": "YI", "YY": "-XZ", "YZ": "XY",
        "ZI": "ZI", "ZX": "ZX", "ZY": "IY", "ZZ": "IZ"}


@pytest.mark.parametrize("inp", sorted(CNOT))
def test_cnot_truth_table(impl, inp):
    assert to_str(impl.apply_cnot(planes([(inp, 1.0)]), 0, 1), 2) == f"1.000000 * {CNOT[inp]}\n"


def test_cnot_high_and_cross_word(impl):
    s = impl.apply_cnot(planes([("IIIIIIIIXIIIIIII", 1.0)]), 8, 9)
    assert to_str(s, 16) == "1.000000 * IIIIIIIIXXIIIIII\n"
    t = impl.apply_cnot(planes([("IIIIIIIIIZIIIIII", 1.0)]), 8, 9)
    assert to_str(t, 16) == "1.000000 * IIIIIIIIZZIIIIII\n"
    inp = ["I"] * 128
    inp[0] = "X"
    exp = list(inp)
    exp[70] = "X"
    u = impl.apply_cnot(planes([("".join(inp), 1.0)]), 0, 70)
    assert to_str(u, 128) == "1.000000 * " + "".join(exp) + "\n"


# PauliSumTests.cpp:899-983 -- evolve fast paths and general angle.
def _evolve(impl, obs, gen, theta):
    return impl.evolve(planes([(obs, 1.0)]), planes([(gen, theta)]))


def test_evolve_fast_paths(impl):
    assert to_str(_evolve(impl, "X", "Z", 0.0), 1) == "1.000000 * X\n"
    assert to_str(_evolve(impl, "X", "Z", math.pi), 1) == "1.000000 * -X\n"
    assert to_str(_evolve(impl, "X", "Z", math.pi / 2), 1) == "1.000000 * -Y\n"
    assert to_str(_evolve(impl, "X", "Z", -math.pi / 2), 1) == "1.000000 * Y\n"


def test_evolve_general_angle(impl):
    th = math.pi / 3
    out = _evolve(impl, "X", "Z", th)
    assert out.n == 2
    assert to_str(Planes(out.x[:, :1], out.z[:, :1], out.flags[:1], out.val[:1]), 1) \
        == f"{math.cos(th):f} * X\n"
    assert out.val[0] == math.cos(th)
    assert out.val[1] == -math.sin(th)


def test_evolve_commuting_unchanged(impl):
    s = planes([("Z", 2.0)])
    for th in (0.0, 0.3, math.pi / 2, -math.pi / 2, math.pi):
        s = impl.evolve(s, planes([("Z", th)]))
    assert to_str(s, 1) == "2.000000 * Z\n"


# PauliSumTests.cpp:1075-1147 -- canonicalize, cutoff, truncate_weight.
def test_canonicalize_folds_sign(impl):
    out = impl.canonicalize(planes([("XI", 1.0), ("-XI", 0.25), ("ZI", 2.0)]))
    terms = {}
    from paulib_b200 import strings
    for i in range(out.n):
        terms[strings.fmt(out.x[:, i], out.z[:, i], out.flags[i], 2)] = out.val[i]
    assert terms == {"XI": 0.75, "ZI": 2.0}


def test_canonicalize_drops_zeros_keeps_imaginary(impl):
    assert impl.canonicalize(planes([("XI", 1.0), ("-XI", 1.0)])).n == 0
    out = impl.canonicalize(planes([("-iZ", 3.0)]))
    assert to_str(out, 1) == "-3.000000 * iZ\n"


def test_cutoff_and_weight(impl):
    s = planes([("XII", 0.5), ("XYZ", 0.01), ("ZZI", -0.2)])
    s = impl.cutoff(s, 0.05)
    assert s.n == 2
    s = impl.truncate_weight(s, 1)
    assert to_str(s, 3) == "0.500000 * XII\n"


# GpuPauliSumTests.cpp:339-343 -- commuting inputs give an empty commutator.
def test_commutator_commuting_empty(impl):
    assert impl.commutator(planes([("ZI", 1.0)]), planes([("IZ", 1.0)])).n == 0


# The reference's i[.,.] shifts the phase exponent by one
# (PauliSumOperations.h:336-337): [X, Z] = 2 XZ = -2i Y.
def test_commutator_values(impl):
    c = impl.commutator(planes([("X", 1.5)]), planes([("Z", 2.0)]))
    assert to_str(c, 1) == "6.000000 * -iY\n"
    ic = impl.commutator(planes([("X", 1.5)]), planes([("Z", 2.0)]), mul_i=True)
    assert to_str(ic, 1) == "6.000000 * Y\n"


# PauliSumTests.cpp:1113-1137 -- trim keeps the largest |c|; a keep set
# protects its patterns and the rest share what is left of the budget.
def _terms(impl_out, nq):
    from paulib_b200 import strings
    return {strings.fmt(impl_out.x[:, i], impl_out.z[:, i], impl_out.flags[i], nq):
            float(impl_out.val[i]) for i in range(impl_out.n)}


def test_trim_keeps_largest(impl):
    s = planes([("XI", 0.1), ("ZI", -5.0), ("IZ", 0.3), ("YI", 2.0)])
    assert _terms(impl.trim(s, 2), 2) == {"ZI": -5.0, "YI": 2.0}


def test_trim_protects_keep_patterns(impl):
    s = planes([("XI", 0.001), ("ZI", -5.0), ("IZ", 0.3), ("YI", 2.0)])
    keep = planes([("XI", 1.0)])
    assert _terms(impl.trim_protected(s, 2, keep), 2) == {"XI": 0.001, "ZI": -5.0}
