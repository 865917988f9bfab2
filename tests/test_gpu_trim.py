"""GPU trim (pl_state_trim / pl_state_trim_protected) and max_terms
truncation against the oracle, through the C ABI.

Survivors and their order are bit-exact: the oracle and the GPU both keep
the largest |c| and break ties at the boundary by lower index.  Inputs with
many equal magnitudes (ties spread over many tiles) exercise that rule.
"""
import numpy as np
import pytest

from helpers import assert_keys_equal, bit_identical, planes, random_sum, to_str
from paulib_b200.planes import Planes
from paulib_b200 import propagation as PR
from paulib_b200 import workloads as W

pytestmark = pytest.mark.gpu


def state_of(p: Planes):
    st = PR.State(p.array_size, max(p.n, 1 << 16))
    st.upload(p.x, p.z, p.flags, p.val)
    return st


def gpu_trim(p, m, keep=None):
    with state_of(p) as st:
        if keep is None:
            st.trim(m)
        else:
            with state_of(keep) as k:
                st.trim(m, k)
        return Planes(*st.download())


def test_golden(cuda):
    # PauliSumTests.cpp:1113-1137
    s = planes([("XI", 0.1), ("ZI", -5.0), ("IZ", 0.3), ("YI", 2.0)])
    assert to_str(gpu_trim(s, 2), 2) == "-5.000000 * ZI\n2.000000 * YI\n"
    s = planes([("XI", 0.001), ("ZI", -5.0), ("IZ", 0.3), ("YI", 2.0)])
    out = gpu_trim(s, 2, planes([("XI", 1.0)]))
    assert to_str(out, 2) == "0.001000 * XI\n-5.000000 * ZI\n"


@pytest.mark.parametrize("n,m,ties", [(1000, 400, False), (200000, 77777, False),
                                      (300000, 150001, True), (50000, 60000, False),
                                      (40000, 0, False), (123457, 1, True)])
def test_random(cuda, oracle, n, m, ties):
    p = random_sum(n, 1, n + m, 40, "normal")
    if ties:  # a handful of magnitudes, both signs: long runs of equal |c|
        rng = np.random.default_rng(5)
        p.val[:] = rng.choice([0.5, 0.25, 0.125, 1e-3], size=n) * rng.choice([-1.0, 1.0], size=n)
    g, o = gpu_trim(p, m), oracle.trim(p, m)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


@pytest.mark.parametrize("words", [1, 2, 4])
def test_protected(cuda, oracle, words):
    p = random_sum(30000, words, 7 * words, None, "normal")
    sel = slice(3, None, 211)
    keep = Planes(p.x[:, sel].copy(), p.z[:, sel].copy(), p.flags[sel].copy(),
                  np.ones(p.x[:, sel].shape[1]))
    for m in (10, 5000, 29999):
        g, o = gpu_trim(p, m, keep), oracle.trim_protected(p, m, keep)
        assert_keys_equal(g, o)
        assert bit_identical(g, o)


def test_propagation_with_max_terms(cuda, oracle):
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=12, layers=4)
    P = lambda s: Planes(s.x, s.z, s.flags, s.val)
    for max_terms in (50, 300):
        o = oracle.propagate(P(obs), P(circ.rotations), circ.ops, max_weight=tr["max_weight"],
                             cutoff=tr["cutoff"], max_terms=max_terms)
        with state_of(P(obs)) as st:
            r = circ.rotations
            st.propagate(r.x, r.z, r.flags, r.val, circ.ops, tr["max_weight"], tr["cutoff"],
                         max_terms)
            g = Planes(*st.download())
        assert_keys_equal(g, o)
        assert bit_identical(g, o)


def test_apply_truncation_with_max_terms(cuda, oracle):
    p = random_sum(20000, 1, 3, 14, "normal")
    with state_of(p) as st:
        st.apply_truncation(max_weight=6, cutoff=1e-3, max_terms=900)
        g = Planes(*st.download())
    o = oracle.trim(oracle.cutoff(oracle.truncate_weight(oracle.canonicalize(p), 6), 1e-3), 900)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)
