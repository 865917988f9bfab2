"""basis_state_expectation, trace, lookup, frobenius_norm2, trace_product:
the C restatement against the reference's own known answers
(PauliSumTests.cpp:715-820, 1041-1070, 1148-1155) and against the reference
build on seeded sums."""
import numpy as np
import pytest

from helpers import planes, random_sum
from paulib_b200 import strings


def words(bits: str, aw: int):
    w = np.zeros(aw, np.uint64)
    for q, ch in enumerate(bits):
        if ch == "1":
            w[q // 64] |= np.uint64(1) << np.uint64(q % 64)
    return w


def test_basis_state_known_answers(oracle):
    s = planes([("II", 1.5), ("ZI", 2.0), ("ZZ", 4.0), ("XI", 8.0), ("IY", 16.0)])
    assert oracle.basis_state_expectation(s, words("00", 1)) == oracle.zero_state_expectation(s)
    s = planes([("ZI", 2.0), ("IZ", 3.0), ("ZZ", 4.0)])
    assert oracle.basis_state_expectation(s, words("10", 1)) == -2.0 + 3.0 - 4.0
    assert oracle.basis_state_expectation(s, words("01", 1)) == 2.0 - 3.0 - 4.0
    assert oracle.basis_state_expectation(s, words("11", 1)) == -2.0 - 3.0 + 4.0
    assert oracle.basis_state_expectation(planes([("XI", 8.0), ("IY", 16.0)]),
                                          words("11", 1)) == 0.0
    assert oracle.basis_state_expectation(planes([("-Z", 3.0), ("Z", 1.0)]), words("1", 1)) == 2.0
    assert oracle.basis_state_expectation(planes([("iZ", 3.0), ("-iZ", 5.0), ("I", 1.0)]),
                                          words("1", 1)) == 1.0


def _lk(oracle, s, q):
    x, z, f, _ = strings.parse(q, s.array_size)
    return oracle.lookup(s, np.array(x, np.uint64), np.array(z, np.uint64), f)


def test_lookup_known_answers(oracle):
    s = planes([("XXII", 1.0), ("IZZI", -0.5), ("IIXY", 0.25)])
    assert (_lk(oracle, s, "XXII"), _lk(oracle, s, "IZZI"), _lk(oracle, s, "IIXY")) == \
        (1.0, -0.5, 0.25)
    s = planes([("XX", 1.0), ("ZI", 2.0)])
    assert _lk(oracle, s, "IZ") == 0.0 and _lk(oracle, s, "YY") == 0.0
    assert _lk(oracle, planes([("XZ", 1.0), ("IY", 4.0), ("XZ", 2.0)]), "XZ") == 3.0
    s = planes([("X", 1.0), ("-X", 0.25), ("iY", 2.0)])
    assert [_lk(oracle, s, q) for q in ("X", "-X", "iY", "-iY")] == [0.75, -0.75, 2.0, -2.0]
    s = planes([("iZ", 3.0), ("Z", 1.0)])
    assert _lk(oracle, s, "Z") == 1.0 and _lk(oracle, s, "iZ") == 3.0
    a, b = ["I"] * 100, ["I"] * 100
    a[3], a[97], b[97] = "X", "Z", "Z"
    a, b = "".join(a), "".join(b)
    s = planes([(a, 1.5), (b, -2.0)])
    assert _lk(oracle, s, a) == 1.5 and _lk(oracle, s, b) == -2.0


def test_trace_and_products_known_answers(oracle):
    s = planes([("IIII", 2.5), ("XIZI", 7.0), ("-IIII", 1.0), ("iIIII", 3.0)])
    assert oracle.trace(s, 4) == 16.0 * 1.5
    assert oracle.trace(planes([("XYZI", 1.0), ("ZZZZ", -3.0)]), 4) == 0.0
    a, b = planes([("XYZ", 1.0)]), planes([("XYI", 1.0)])
    assert oracle.trace_product(a, a, 3) == 8.0 and oracle.trace_product(a, b, 3) == 0.0
    s = oracle.canonicalize(planes([("XII", 0.5), ("ZZI", -0.2), ("XYZ", 1.5)]))
    assert abs(oracle.frobenius_norm2(s) - oracle.trace_product(s, s, 3) / 8.0) <= 1e-14


@pytest.mark.parametrize("words_", [1, 2])
def test_reductions_match_reference(oracle, reference, words_):
    nq = 64 * words_
    s = random_sum(3000, words_, 5 + words_, 12, "normal")   # few qubits: many I/Z terms
    bits = np.array([0x5a5a5a5a5a5a5a5a] * words_, np.uint64)
    for fn, args in ((oracle.basis_state_expectation, (bits,)), ):
        assert abs(fn(s, *args) - reference.basis_state_expectation(s, bits)) <= 1e-9
    assert abs(oracle.trace(s, nq) - reference.trace(s, nq)) <= 1e-12 * abs(reference.trace(s, nq)) + 1e-300
    assert abs(oracle.frobenius_norm2(s) - reference.frobenius_norm2(s)) <= 1e-9
    q = s.x[:, 7], s.z[:, 7], int(s.flags[7])
    assert abs(oracle.lookup(s, *q) - reference.lookup(s, *q)) <= 1e-12
    t = random_sum(2000, words_, 9 + words_, 12, "normal")
    got, ref = oracle.trace_product(s, t, nq), reference.trace_product(s, t, nq)
    assert abs(got - ref) <= 1e-9 * max(1.0, abs(ref))
