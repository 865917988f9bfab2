"""GPU bulk Clifford gates (pl_state_apply_clifford), rotation gates
(pl_state_apply_rotation_gate) and Clifford ops inside pl_propagate,
against the reference's known answers and the oracle, through the C ABI.

Cliffords are bijections of the strings that keep term order and
coefficients: everything bit-exact.  Rotation gates merge at most two
contributions per key (old and child), so coefficients are bit-exact too."""
import math

import numpy as np
import pytest

from gates_golden import GATE, ONE_QUBIT, ROTATIONS, TWO_QUBIT
from helpers import assert_keys_equal, bit_identical, planes, random_sum, to_str
from paulib_b200.planes import Planes
from paulib_b200 import propagation as PR
from paulib_b200 import workloads as W

pytestmark = pytest.mark.gpu


def on_gpu(p: Planes, fn):
    with PR.State(p.array_size, max(p.n, 1 << 16)) as st:
        st.upload(p.x, p.z, p.flags, p.val)
        fn(st)
        return Planes(*st.download())


@pytest.mark.parametrize("gate", sorted(ONE_QUBIT))
def test_one_qubit_truth_tables(cuda, gate):
    for inp, out in ONE_QUBIT[gate].items():
        g = on_gpu(planes([(inp, 1.0)]), lambda st: st.apply_clifford(GATE[gate], 0))
        assert to_str(g, 1) == f"1.000000 * {out}\n", (gate, inp)


@pytest.mark.parametrize("gate", sorted(TWO_QUBIT))
def test_two_qubit_truth_tables(cuda, gate):
    for inp, out in TWO_QUBIT[gate].items():
        g = on_gpu(planes([(inp, 1.0)]), lambda st: st.apply_clifford(GATE[gate], 0, 1))
        assert to_str(g, 2) == f"1.000000 * {out}\n", (gate, inp)


def test_iswap_known_answer(cuda):
    g = on_gpu(planes([("XI", 1.0)]), lambda st: st.apply_clifford(GATE["ISWAP"], 0, 1))
    assert to_str(g, 2) == "1.000000 * ZY\n"


@pytest.mark.parametrize("words,pairs", [(1, [(3, 40), (40, 3), (0, 63)]),
                                         (2, [(5, 100), (100, 5), (70, 71)]),
                                         (3, [(10, 150), (129, 2)])])
def test_random_sums_match_oracle(cuda, oracle, words, pairs):
    p = random_sum(5000, words, 11 * words, None, "normal")
    for gate in range(1, 22):
        for c, t in pairs:
            g = on_gpu(p, lambda st: st.apply_clifford(gate, c, t))
            o = oracle.apply_clifford(p, gate, c, t)
            assert_keys_equal(g, o)
            assert bit_identical(g, o), (gate, c, t)


@pytest.mark.parametrize("case", range(len(ROTATIONS)))
def test_rotation_gate_known_answers(cuda, case):
    axis, inp, exp = ROTATIONS[case]
    g = on_gpu(planes(inp), lambda st: st.apply_rotation_gate(axis, 0, math.pi / 3))
    assert to_str(g, 1) == exp


@pytest.mark.parametrize("words", [1, 2])
def test_rotation_gates_match_oracle(cuda, oracle, words):
    p = random_sum(20000, words, 3 + words, 40 if words == 1 else 100, "normal")
    for axis in (1, 2, 3):
        for q, th in ((4, 0.37), (31, 2.9)):
            g = on_gpu(p, lambda st: st.apply_rotation_gate(axis, q, th))
            o = oracle.apply_rgate(p, axis, q, th)
            assert_keys_equal(g, o)
            assert bit_identical(g, o), (axis, q, th)


def test_propagation_with_clifford_ops(cuda, oracle):
    # a brickwork circuit with Clifford layers spliced in
    obs, circ, tr = W.heisenberg_workload(seed=4, num_qubits=12, layers=3)
    ops = []
    rng = np.random.default_rng(9)
    for row in circ.ops:
        ops.append(tuple(int(v) for v in row))
        if rng.random() < 0.15:
            g = int(rng.integers(1, 22))
            a, b = (int(v) for v in rng.choice(12, size=2, replace=False))
            ops.append((100 + g, a, b))
    ops = np.asarray(ops, np.int32)
    P = lambda s: Planes(s.x, s.z, s.flags, s.val)
    o = oracle.propagate(P(obs), P(circ.rotations), ops, max_weight=tr["max_weight"],
                         cutoff=tr["cutoff"])
    r = circ.rotations

    def run(st):
        st.propagate(r.x, r.z, r.flags, r.val, ops, tr["max_weight"], tr["cutoff"])

    g = on_gpu(P(obs), run)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_python_surface_gates(cuda):
    from paulib_b200 import paulib as PL
    s = PL.PauliSum([("IZXY", 1.0)])
    for q in range(4):
        s.apply_H(q)
    assert str(s) == "1.000000 * -IXZY\n"
    t = PL.PauliSum([("Z", 2.0), ("X", 1.0)])
    t.apply_RZ(0, math.pi / 3)
    assert str(t) == "2.000000 * Z\n0.866025 * X\n0.500000 * -Y\n"
    with pytest.raises(ValueError):
        PL.PauliSum([("XX", 1.0)]).apply_CZ(1, 1)
