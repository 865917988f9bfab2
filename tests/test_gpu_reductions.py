"""GPU reductions (pl_state_basis_state_expectation / trace / lookup /
frobenius_norm2 / trace_product) against the reference's known answers and
the oracle.  The GPU sums in a fixed parallel order, the reference in term
order: results agree within 1e-12 of the summed magnitudes (exact on the
known-answer cases)."""
import numpy as np
import pytest

from helpers import planes, random_sum
from paulib_b200 import paulib as PL
from paulib_b200 import propagation as PR
from paulib_b200 import strings
from paulib_b200.planes import Planes

pytestmark = pytest.mark.gpu


def state_of(p: Planes):
    st = PR.State(p.array_size, max(p.n, 1 << 16))
    st.upload(p.x, p.z, p.flags, p.val)
    return st


def test_known_answers(cuda):
    s = PL.PauliSum([("II", 1.5), ("ZI", 2.0), ("ZZ", 4.0), ("XI", 8.0), ("IY", 16.0)])
    assert s.basis_state_expectation("00") == s.zero_state_expectation()
    s = PL.PauliSum([("ZI", 2.0), ("IZ", 3.0), ("ZZ", 4.0)])
    assert s.basis_state_expectation("10") == -2.0 + 3.0 - 4.0
    assert s.basis_state_expectation("01") == 2.0 - 3.0 - 4.0
    assert s.basis_state_expectation("11") == -2.0 - 3.0 + 4.0
    assert PL.PauliSum([("-Z", 3.0), ("Z", 1.0)]).basis_state_expectation("1") == 2.0
    assert PL.PauliSum([("iZ", 3.0), ("-iZ", 5.0), ("I", 1.0)]).basis_state_expectation("1") == 1.0
    with pytest.raises(ValueError):
        s.basis_state_expectation("0")
    with pytest.raises(ValueError):
        s.basis_state_expectation("02")
    l = PL.PauliSum([("X", 1.0), ("-X", 0.25), ("iY", 2.0)])
    assert [l.lookup(q) for q in ("X", "-X", "iY", "-iY")] == [0.75, -0.75, 2.0, -2.0]
    assert PL.PauliSum([("XZ", 1.0), ("IY", 4.0), ("XZ", 2.0)]).lookup("XZ") == 3.0
    assert PL.PauliSum([("XX", 1.0), ("ZI", 2.0)]).lookup("YY") == 0.0
    t = PL.PauliSum([("IIII", 2.5), ("XIZI", 7.0), ("-IIII", 1.0), ("iIIII", 3.0)])
    assert t.trace() == 16.0 * 1.5
    assert PL.PauliSum([("XYZI", 1.0), ("ZZZZ", -3.0)]).trace() == 0.0
    a, b = PL.PauliSum([("XYZ", 1.0)]), PL.PauliSum([("XYI", 1.0)])
    assert PL.trace_product(a, a) == 8.0 and PL.trace_product(a, b) == 0.0
    with pytest.raises(ValueError):
        PL.trace_product(a, PL.PauliSum([("XYZI", 1.0)]))
    c = PL.PauliSum([("XII", 0.5), ("ZZI", -0.2), ("XYZ", 1.5)])
    c.canonicalize()
    assert abs(c.frobenius_norm2() - PL.trace_product(c, c) / 8.0) <= 1e-14


@pytest.mark.parametrize("words", [1, 2, 4])
def test_match_oracle(cuda, oracle, words):
    nq = 64 * words
    p = random_sum(100000, words, 20 + words, 14, "normal")   # many I / Z terms
    q = random_sum(60000, words, 30 + words, 14, "normal")
    mag = float(np.abs(p.val).sum())
    bits = np.array([0x0123456789abcdef] * words, np.uint64)
    with state_of(p) as sp, state_of(q) as sq:
        assert abs(sp.basis_state_expectation(bits) -
                   oracle.basis_state_expectation(p, bits)) <= 1e-12 * mag
        assert abs(sp.trace(nq) - oracle.trace(p, nq)) <= 1e-12 * mag * 2.0 ** nq
        assert abs(sp.frobenius_norm2() - oracle.frobenius_norm2(p)) <= \
            1e-12 * float((p.val ** 2).sum())
        for i in (0, 17, 999):
            x, z, f = p.x[:, i], p.z[:, i], int(p.flags[i])
            assert abs(sp.lookup(x, z, f) - oracle.lookup(p, x, z, f)) <= 1e-12 * mag
    # the oracle's trace_product scans A for every term of B: smaller sums
    a, b = random_sum(4000, words, 40 + words, 10, "normal"), random_sum(3000, words, 50, 10,
                                                                          "normal")
    with state_of(a) as sa, state_of(b) as sb:
        got = sa.trace_product(sb, nq)
    ref = oracle.trace_product(a, b, nq)
    scale = float(np.abs(a.val).sum()) * float(np.abs(b.val).sum()) * 2.0 ** nq
    assert abs(got - ref) <= 1e-12 * scale
