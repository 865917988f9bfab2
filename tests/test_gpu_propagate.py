"""GPU parity of the device-resident propagation (pl_state_*, pl_propagate)
against the oracle and the reference build, through the C ABI.

Each canonical key receives at most two contributions per rotation, so the
propagated sums -- strings, phases, order and coefficients -- must be
bit-identical to the reference; the final zero_state_expectation is a
parallel reduction and must agree within 1e-10 absolute.
"""
import math

import numpy as np
import pytest

from gpu_util import as_planes
from helpers import (abs_scale, assert_keys_equal, assert_values_close, bit_identical, planes,
                     random_sum, to_str)
from paulib_b200.planes import Planes
from paulib_b200 import propagation as PR
from paulib_b200 import workloads as W

pytestmark = pytest.mark.gpu


def state_of(p: Planes, hint=1 << 16):
    st = PR.State(p.array_size, hint)
    st.upload(p.x, p.z, p.flags, p.val)
    return st


def planes_of(st) -> Planes:
    return Planes(*st.download())


def gpu_evolve(p: Planes, rot: Planes) -> Planes:
    with state_of(p) as st:
        st.evolve(rot.x, rot.z, rot.flags, rot.val)
        return planes_of(st)


# PauliSumTests.cpp:899-983 -- evolve fast paths and the general angle.
@pytest.mark.parametrize("theta,expect", [(0.0, "1.000000 * X\n"), (math.pi, "1.000000 * -X\n"),
                                          (math.pi / 2, "1.000000 * -Y\n"),
                                          (-math.pi / 2, "1.000000 * Y\n")])
def test_evolve_fast_paths(cuda, theta, expect):
    assert to_str(gpu_evolve(planes([("X", 1.0)]), planes([("Z", theta)])), 1) == expect


def test_evolve_general(cuda, oracle):
    th = math.pi / 3
    g = gpu_evolve(planes([("X", 1.0)]), planes([("Z", th)]))
    assert g.n == 2 and g.val[0] == math.cos(th) and g.val[1] == -math.sin(th)
    o = oracle.evolve(planes([("X", 1.0)]), planes([("Z", th)]))
    assert_keys_equal(g, o)


def test_evolve_commuting_unchanged(cuda):
    s = planes([("Z", 2.0)])
    for th in (0.0, 0.3, math.pi / 2, -math.pi / 2, math.pi):
        s = gpu_evolve(s, planes([("Z", th)]))
    assert to_str(s, 1) == "2.000000 * Z\n"


@pytest.mark.parametrize("words,nq", [(1, 40), (2, 100)])
def test_evolve_random_noncanonical(cuda, oracle, words, nq):
    s = random_sum(400, words, 11, nq)  # random flags, duplicates possible
    rot = random_sum(7, words, 12, nq, "normal", flags="zero")
    rot.val[2] = math.pi
    rot.val[4] = math.pi / 2
    g, o = gpu_evolve(s, rot), oracle.evolve(s, rot)
    assert_keys_equal(g, o)
    assert_values_close(g, o, abs_scale(oracle, s))


def test_state_ops_match_oracle(cuda, oracle):
    p = random_sum(5000, 1, 3, 12, "normal")
    with state_of(p) as st:
        st.canonicalize()
        g = planes_of(st)
    o = oracle.canonicalize(p)
    assert_keys_equal(g, o)
    assert_values_close(g, o, abs_scale(oracle, p))
    with state_of(p) as st:
        st.sort_and_combine()
        g = planes_of(st)
    o2 = oracle.sort_and_combine(p)
    assert_keys_equal(g, o2)
    with state_of(o) as st:
        st.truncate_weight(5)
        st.cutoff(0.5)
        st.apply_cnot(3, 7)
        g = planes_of(st)
        e = st.zero_state_expectation()
    o3 = oracle.apply_cnot(oracle.cutoff(oracle.truncate_weight(o, 5), 0.5), 3, 7)
    assert_keys_equal(g, o3)
    assert bit_identical(g, o3)
    assert abs(e - oracle.zero_state_expectation(o3)) <= 1e-10


@pytest.mark.parametrize("nq,layers", [(12, 4), (20, 3), (64, 3), (64, 4)])
def test_brickwork_matches_oracle(cuda, oracle, nq, layers):
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=nq, layers=layers)
    kw = dict(max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    o = oracle.propagate(as_planes(obs), as_planes(circ.rotations), circ.ops, **kw)
    with state_of(as_planes(obs)) as st:
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        g = planes_of(st)
        e = st.zero_state_expectation()
    assert_keys_equal(g, o)
    assert bit_identical(g, o)
    assert abs(e - oracle.zero_state_expectation(o)) <= 1e-10


def test_brickwork_grows_buffers(cuda, reference):
    # 64 qubits, 5 layers: the sum passes 65536 terms, so the state must
    # detect the overflow on the device, grow and replay.
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=64, layers=5)
    kw = dict(max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    ref = reference.propagate(as_planes(obs), as_planes(circ.rotations), circ.ops, **kw)
    with state_of(as_planes(obs), hint=1024) as st:
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        g = planes_of(st)
        e = st.zero_state_expectation()
    assert_keys_equal(g, ref)
    assert bit_identical(g, ref)
    assert abs(e - reference.zero_state_expectation(ref)) <= 1e-10


def test_wide_strings(cuda, oracle):
    # 100 qubits (2 words), CNOTs across the word boundary
    obs, circ, tr = W.heisenberg_workload(seed=5, num_qubits=100, layers=2)
    kw = dict(max_weight=6, cutoff=1e-3)
    o = oracle.propagate(as_planes(obs), as_planes(circ.rotations), circ.ops, **kw)
    with state_of(as_planes(obs)) as st:
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        g = planes_of(st)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_fast_path_angles_in_circuit(cuda, oracle):
    obs, circ, tr = W.heisenberg_workload(seed=9, num_qubits=16, layers=3)
    th = circ.rotations.val
    th[::7] = math.pi
    th[1::11] = math.pi / 2
    th[2::13] = -math.pi / 2
    th[3::17] = 0.0
    kw = dict(max_weight=8, cutoff=1e-4)
    o = oracle.propagate(as_planes(obs), as_planes(circ.rotations), circ.ops, **kw)
    with state_of(as_planes(obs)) as st:
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        g = planes_of(st)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_rotation_only_any_generators(cuda, oracle):
    # The reference's own propagate(): multi-qubit generators take the
    # general path; the observable is not canonical on entry.
    obs = random_sum(5, 1, 21, 10, "normal")
    rot = random_sum(25, 1, 22, 10, "normal", flags="zero")
    o = oracle.propagate(obs, rot, None, max_weight=6, cutoff=1e-3)
    with state_of(obs) as st:
        st.propagate(rot.x, rot.z, rot.flags, rot.val, None, max_weight=6, cutoff=1e-3)
        g = planes_of(st)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_expectation_helper(cuda, oracle):
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=10, layers=3)
    e = PR.propagate_expectation_planes(obs, circ, tr["max_weight"], tr["cutoff"])
    o = oracle.propagate(as_planes(obs), as_planes(circ.rotations), circ.ops,
                         max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    assert abs(e - oracle.zero_state_expectation(o)) <= 1e-10


# ---------------------------------------------------------------------------
# algebra on device-resident states (pl_state_multiply / _canonicalize /
# pl_state_commutator)
# ---------------------------------------------------------------------------
def test_state_multiply(cuda, oracle):
    import ctypes
    from paulib_b200 import _abi
    a, b = random_sum(37, 2, 1, 100), random_sum(23, 2, 2, 100, "normal")
    with state_of(a, hint=8) as sa, state_of(b, hint=8) as sb:
        _abi.check(_abi.lib().pl_state_multiply(sa._h, sb._h))
        g = planes_of(sa)
    o = oracle.multiply(a, b)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_state_multiply_canonicalize(cuda, oracle):
    from paulib_b200 import _abi
    a, b = W.product_operands(seed=5, terms=300)
    a, b = as_planes(a), as_planes(b)
    with state_of(a, hint=16) as sa, state_of(b, hint=16) as sb:
        _abi.check(_abi.lib().pl_state_multiply_canonicalize(sa._h, sb._h))
        g = planes_of(sa)
    prod = oracle.multiply(a, b)
    o = oracle.canonicalize(prod)
    assert_keys_equal(g, o)
    assert_values_close(g, o, abs_scale(oracle, prod))


@pytest.mark.parametrize("mul_i", [0, 1])
def test_state_commutator(cuda, oracle, mul_i):
    from paulib_b200 import _abi
    a, b = W.window_sums(seed=4, terms=700)
    a, b = as_planes(a), as_planes(b)
    with state_of(a) as sa, state_of(b) as sb, PR.State(4, 16) as so:
        _abi.check(_abi.lib().pl_state_commutator(so._h, sa._h, sb._h, mul_i))
        g = planes_of(so)
    o = oracle.commutator(a, b, bool(mul_i))
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_gate_log_sizes(cuda, oracle):
    # PL_OPT_GATE_LOG: per fast-path rotation (terms in, anticommuting,
    # terms out), in processing order; logging changes no result.
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=20, layers=3)
    kw = dict(max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    r = circ.rotations
    with state_of(as_planes(obs)) as st:
        st.use_graphs(True).log_gates(True)
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        g = planes_of(st)
        log = st.gate_log()
    o = oracle.propagate(as_planes(obs), as_planes(r), circ.ops, **kw)
    assert bit_identical(g, o)
    assert log.shape == (circ.ops.shape[0], 3)
    rot_rows = circ.ops[::-1, 0] == W.OP_ROT
    assert (log[~rot_rows] == 0).all()
    rows = log[rot_rows]
    # every rotation of this circuit takes the fast path
    assert (rows[:, 0] > 0).all()
    assert rows[0, 0] == obs.n and rows[-1, 2] == g.n
    # CNOT layers keep the size: each rotation starts from the last one's output
    assert np.array_equal(rows[1:, 0], rows[:-1, 2])
    assert (rows[:, 1] <= rows[:, 0]).all()
    assert (rows[:, 2] <= rows[:, 0] + rows[:, 1]).all()
