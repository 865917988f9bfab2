"""The C restatement against the reference's own implementation (compiled
from the reference headers into oracle/_ref/) on seeded random cases.

Strings, phases and term order must agree bit for bit.  Coefficients of
multiply / commutator / evolve / propagation agree bit for bit as well; the
collate coefficients are compared within 1e-12 of the summed magnitudes,
because the reference build (-ffast-math) reassociates its segment-sum loop
(PauliSumOperations.h:453) while the restatement sums strictly left to right.
"""
import numpy as np
import pytest

from helpers import abs_scale, assert_keys_equal, assert_values_close, bit_identical, random_sum
from paulib_b200 import workloads as W
from paulib_b200.planes import Planes


def P(s):
    return Planes(s.x, s.z, s.flags, s.val)


@pytest.mark.parametrize("words", [1, 2, 4])
def test_multiply(oracle, reference, words):
    a, b = random_sum(37, words, 1), random_sum(23, words, 2)
    o, r = oracle.multiply(a, b), reference.multiply(a, b)
    assert_keys_equal(o, r)
    assert bit_identical(o, r)


@pytest.mark.parametrize("words", [1, 3])
def test_canonicalize_product(oracle, reference, words):
    a, b = W.product_operands(seed=7, terms=200) if words == 1 else \
        (random_sum(150, words, 5, 70, "normal"), random_sum(140, words, 6, 70, "normal"))
    prod = oracle.multiply(P(a) if words == 1 else a, P(b) if words == 1 else b)
    o, r = oracle.canonicalize(prod), reference.canonicalize(prod)
    assert_keys_equal(o, r)
    assert_values_close(o, r, abs_scale(oracle, prod))


def test_sort_and_combine_product(oracle, reference):
    a, b = W.product_operands(seed=8, terms=150)
    prod = oracle.multiply(P(a), P(b))
    o, r = oracle.sort_and_combine(prod), reference.sort_and_combine(prod)
    assert_keys_equal(o, r)
    assert_values_close(o, r, abs_scale(oracle, prod))


def test_commutator_single_thread_order(oracle, reference):
    a, b = W.window_sums(seed=3, terms=500)
    reference.set_threads(1)  # the multithreaded CPU commutator's order is nondeterministic
    try:
        o, r = oracle.commutator(P(a), P(b)), reference.commutator(P(a), P(b))
    finally:
        reference.set_threads(reference.lib.ref_max_threads())
    assert_keys_equal(o, r)
    assert bit_identical(o, r)
    co = oracle.cutoff(oracle.canonicalize(o), 1e-14)
    cr = reference.cutoff(reference.canonicalize(r), 1e-14)
    assert_keys_equal(co, cr)
    assert_values_close(co, cr, abs_scale(oracle, o))


def test_evolve_random(oracle, reference):
    s = random_sum(300, 1, 11, 40)
    rot = random_sum(6, 1, 12, 40, "normal", flags="zero")
    o, r = oracle.evolve(s, rot), reference.evolve(s, rot)
    assert_keys_equal(o, r)
    assert_values_close(o, r, abs_scale(oracle, s), rtol=1e-12)


@pytest.mark.parametrize("nq,layers", [(12, 4), (20, 3)])
def test_propagation_brickwork(oracle, reference, nq, layers):
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=nq, layers=layers)
    kw = dict(max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    o = oracle.propagate(P(obs), P(circ.rotations), circ.ops, **kw)
    r = reference.propagate(P(obs), P(circ.rotations), circ.ops, **kw)
    assert_keys_equal(o, r)
    assert bit_identical(o, r)
    assert oracle.zero_state_expectation(o) == reference.zero_state_expectation(r)


def test_propagation_rotation_only(oracle, reference):
    # The reference's own propagate(): rotations only, any generators.
    obs = random_sum(3, 1, 21, 10, "normal", flags="zero")
    rot = random_sum(25, 1, 22, 10, "normal", flags="zero")
    o = oracle.propagate(obs, rot, None, max_weight=6, cutoff=1e-3)
    r = reference.propagate(obs, rot, None, max_weight=6, cutoff=1e-3)
    assert_keys_equal(o, r)
    assert bit_identical(o, r)


@pytest.mark.parametrize("words,n,m", [(1, 3000, 1000), (2, 2000, 1999), (4, 500, 10)])
def test_trim(oracle, reference, words, n, m):
    # N(0,1) coefficients: no ties at the boundary, so nth_element's choice
    # and the restatement's lower-index rule pick the same terms
    s = random_sum(n, words, 31 + words, None, "normal")
    o, r = oracle.trim(s, m), reference.trim(s, m)
    assert_keys_equal(o, r)
    assert bit_identical(o, r)


def test_trim_protected(oracle, reference):
    s = random_sum(2000, 1, 41, 30, "normal")
    keep = Planes(s.x[:, ::97].copy(), s.z[:, ::97].copy(), s.flags[::97].copy(),
                  np.ones(s.x[:, ::97].shape[1]))
    o, r = oracle.trim_protected(s, 300, keep), reference.trim_protected(s, 300, keep)
    assert_keys_equal(o, r)
    assert bit_identical(o, r)
