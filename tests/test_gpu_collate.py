"""GPU parity of the collate engine (canonicalize / sort_and_combine /
cutoff / truncate_weight, and the fused product + canonicalize) against the
oracle, through the C ABI.

Strings, phases and order: bit-exact.  Coefficients: every segment of at
most 32 contributions is summed in the reference's left-to-right order, so
it is bit-identical to the strict oracle; longer segments use a fixed-order
parallel sum and must agree within 1e-12 of their summed magnitudes.
"""
import numpy as np
import pytest

from gpu_util import as_planes, gpu_collate, gpu_multiply_collate
from helpers import (abs_scale, assert_keys_equal, assert_values_close, bit_identical, planes,
                     random_sum, to_str)
from paulib_b200.planes import Planes
from paulib_b200 import _abi
from paulib_b200 import workloads as W

pytestmark = pytest.mark.gpu
CANON = _abi.PL_COLLATE_CANONICALIZE
COMBINE = _abi.PL_COLLATE_SORT_AND_COMBINE


def _check(g, o, inp, oracle, exact=False):
    assert_keys_equal(g, o)
    if exact:
        assert bit_identical(g, o)
    else:
        assert_values_close(g, o, abs_scale(oracle, inp))


def test_golden_small(cuda):
    # PauliSumTests.cpp:514-561, 1083-1115.
    out = gpu_collate(planes([("XY", 2.0), ("ZZ", 1.0), ("XY", 3.0)]), COMBINE)
    assert to_str(out, 2) == "1.000000 * ZZ\n5.000000 * XY\n"
    out = gpu_collate(planes([("X", 2.0), ("-X", 3.0)]), COMBINE)
    assert to_str(out, 1) == "2.000000 * X\n3.000000 * -X\n"
    out = gpu_collate(planes([("X", 2.0), ("X", -2.0)]), COMBINE)
    assert out.n == 1 and out.val[0] == 0.0
    assert gpu_collate(planes([("XI", 1.0), ("-XI", 1.0)]), CANON).n == 0
    assert to_str(gpu_collate(planes([("-iZ", 3.0)]), CANON), 1) == "-3.000000 * iZ\n"
    s = gpu_collate(planes([("XII", 0.5), ("XYZ", 0.01), ("ZZI", -0.2)]), CANON, cutoff=0.05,
                    max_weight=1)
    assert to_str(s, 3) == "0.500000 * XII\n"


def test_empty_and_single(cuda):
    assert gpu_collate(Planes.empty(1, 0)).n == 0
    assert to_str(gpu_collate(planes([("Y", 1.5)]), COMBINE), 1) == "1.500000 * Y\n"


@pytest.mark.parametrize("mode", [CANON, COMBINE])
@pytest.mark.parametrize("words,n,nq", [(1, 1000, 8), (1, 50000, 12), (2, 20000, 70),
                                        (4, 30000, 256), (1, 100000, 64), (3, 7777, 150)])
def test_random_sums(cuda, oracle, mode, words, n, nq):
    # few qubits -> many duplicates and long segments; many qubits -> wide keys
    p = random_sum(n, words, n + words, nq, "normal")
    g = gpu_collate(p, mode)
    o = oracle.canonicalize(p) if mode == CANON else oracle.sort_and_combine(p)
    _check(g, o, p, oracle)


def test_short_segments_bit_identical(cuda, oracle):
    # with 16 qubits and 20000 terms every key repeats a handful of times
    p = random_sum(20000, 1, 77, 16, "normal")
    g, o = gpu_collate(p), oracle.canonicalize(p)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


@pytest.mark.parametrize("cutoff,max_weight", [(0.5, None), (0.0, 3), (1e-3, 5)])
def test_filters(cuda, oracle, cutoff, max_weight):
    p = random_sum(40000, 1, 5, 10, "normal")
    g = gpu_collate(p, CANON, cutoff=cutoff, max_weight=max_weight)
    o = oracle.canonicalize(p)
    if max_weight is not None:
        o = oracle.truncate_weight(o, max_weight)
    if cutoff > 0:
        o = oracle.cutoff(o, cutoff)
    _check(g, o, p, oracle)


def test_idempotent(cuda):
    p = random_sum(30000, 2, 9, 80, "normal")
    once = gpu_collate(p)
    twice = gpu_collate(once)
    assert_keys_equal(once, twice)
    assert bit_identical(once, twice)


def test_deterministic(cuda):
    p = random_sum(200000, 1, 19, 14, "normal")
    a, b = gpu_collate(p), gpu_collate(p)
    assert_keys_equal(a, b)
    assert bit_identical(a, b)


def test_capacity_reported(cuda, oracle):
    p = random_sum(5000, 1, 1, 30, "normal")
    n_out = oracle.canonicalize(p).n
    with pytest.raises(_abi.PLError) as e:
        gpu_collate(p, capacity=n_out - 1)
    assert e.value.status == _abi.PL_ERR_CAPACITY


@pytest.mark.parametrize("terms", [64, 700])
def test_multiply_collate_product_workload(cuda, oracle, terms):
    a, b = W.product_operands(seed=terms, terms=terms)
    a, b = as_planes(a), as_planes(b)
    g = gpu_multiply_collate(a, b)
    prod = oracle.multiply(a, b)
    o = oracle.canonicalize(prod)
    _check(g, o, prod, oracle)


@pytest.mark.parametrize("words,n,m,nq", [(2, 300, 200, 100), (4, 120, 90, 256),
                                          (1, 1000, 3, 64)])
def test_multiply_collate_random(cuda, oracle, words, n, m, nq):
    a = random_sum(n, words, 3, nq, "normal")
    b = random_sum(m, words, 4, nq, "normal")
    for mode in (CANON, COMBINE):
        g = gpu_multiply_collate(a, b, mode)
        prod = oracle.multiply(a, b)
        o = oracle.canonicalize(prod) if mode == CANON else oracle.sort_and_combine(prod)
        _check(g, o, prod, oracle)


def test_commutator_workload_collate(cuda, oracle):
    # config-3 shape, reduced: commutator then canonicalize + cutoff(1e-14)
    from gpu_util import gpu_commutator
    a, b = W.window_sums(seed=3, terms=1500)
    a, b = as_planes(a), as_planes(b)
    c = gpu_commutator(a, b)
    g = gpu_collate(c, CANON, cutoff=1e-14)
    oc = oracle.commutator(a, b)
    o = oracle.cutoff(oracle.canonicalize(oc), 1e-14)
    _check(g, o, oc, oracle)


def _windowed(n, nq, seed, lo=2, hi=6):
    from paulib_b200.workloads import window_sums
    a, b = window_sums(seed=seed, terms=n, num_qubits=nq, min_len=lo, max_len=hi)
    return Planes(a.x, a.z, a.flags, a.val), Planes(b.x, b.z, b.flags, b.val)


def _with_window_keys(value, fn):
    from paulib_b200 import _abi
    L = _abi.lib()
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_WINDOW_KEYS, value))
    try:
        return fn()
    finally:
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_WINDOW_KEYS, 0))


@pytest.mark.parametrize("mode", [CANON, COMBINE])
@pytest.mark.parametrize("nq,n", [(256, 40000), (128, 30000), (1000, 20000)])
def test_window_keys_match_plain_layout_and_oracle(cuda, oracle, mode, nq, n):
    # commutator output of windowed sums: products of overlapping windows,
    # every term's support within <= 11 adjacent qubits (PL_TUNE_WINDOW_KEYS)
    a, b = _windowed(1500, nq, seed=n)
    raw = oracle.commutator(a, b)
    rng = np.random.default_rng(n)
    raw = Planes(raw.x, raw.z, rng.integers(0, 4, raw.n).astype(np.uint8), raw.val)
    on = _with_window_keys(0, lambda: gpu_collate(raw, mode))
    off = _with_window_keys(-1, lambda: gpu_collate(raw, mode))
    o = oracle.canonicalize(raw) if mode == CANON else oracle.sort_and_combine(raw)
    assert_keys_equal(on, o)
    assert bit_identical(on, off)
    assert_values_close(on, o, abs_scale(oracle, raw))


def test_window_keys_fall_back_on_wide_supports(cuda, oracle):
    # random strings over 256 qubits do not fit the window form
    p = random_sum(20000, 4, 31, 256, "normal")
    g = _with_window_keys(0, lambda: gpu_collate(p, CANON, cutoff=1e-3))
    o = oracle.cutoff(oracle.canonicalize(p), 1e-3)
    assert_keys_equal(g, o)
    assert_values_close(g, o, abs_scale(oracle, p))
