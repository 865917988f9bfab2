"""GPU parity of canonicalize() on index-packed keys.

When the varying x / z bits of a sum and its term index fit one 64-bit word,
the collate engine sorts (x, z, index) words and keeps the phase out of the
sort key: every (x, z) segment folds its phase-0 and phase-1 members into two
sums, each in index order (PauliSumOperations.h:369-461 with the sign fold of
PauliSumUtils.h:315-328).  Each case here runs with that path allowed and
with it switched off (PL_TUNE_INDEX_KEYS = -1, the general key + payload
sort) and checks both against the oracle and against each other: strings,
phases and order bit-exact; coefficients bit-identical wherever segments are
short, within 1e-12 of the summed magnitudes where long runs use the
fixed-order parallel sum.
"""
import contextlib
import ctypes

import numpy as np
import pytest

from gpu_util import as_planes, gpu_collate, gpu_multiply_collate
from paulib_b200.planes import Planes
from helpers import abs_scale, assert_keys_equal, assert_values_close, bit_identical, random_sum
from paulib_b200 import _abi
from paulib_b200 import workloads as W

pytestmark = pytest.mark.gpu
CANON = _abi.PL_COLLATE_CANONICALIZE


@contextlib.contextmanager
def index_keys(value):
    L = _abi.lib()
    old = ctypes.c_int64()
    _abi.check(L.pl_get_tuning(_abi.PL_TUNE_INDEX_KEYS, ctypes.byref(old)), "pl_get_tuning")
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_INDEX_KEYS, value), "pl_set_tuning")
    try:
        yield
    finally:
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_INDEX_KEYS, old.value), "pl_set_tuning")


def both(fn):
    with index_keys(0):
        on = fn()
    with index_keys(-1):
        off = fn()
    return on, off


def test_tuning_values(cuda):
    L = _abi.lib()
    for bad in (2, -2, 7):
        assert L.pl_set_tuning(_abi.PL_TUNE_INDEX_KEYS, bad) == _abi.PL_ERR_INVALID_ARG
    v = ctypes.c_int64()
    _abi.check(L.pl_get_tuning(_abi.PL_TUNE_INDEX_KEYS, ctypes.byref(v)))
    assert v.value in (0, 1)


@pytest.mark.parametrize("n,nq,seed", [(1, 3, 1), (2, 1, 2), (1000, 8, 3), (50000, 12, 4),
                                       (20000, 16, 5), (4096, 26, 6), (4097, 26, 7),
                                       (300000, 3, 8)])
def test_random_sums(cuda, oracle, n, nq, seed):
    # (4096, 26): 52 x / z bits + 12 index bits fill the word exactly;
    # (4097, 26) needs 65 bits and takes the general path.  nq = 3 with
    # 300000 terms gives segments of several thousand terms (long runs).
    p = random_sum(n, 1, seed, nq, "normal")
    on, off = both(lambda: gpu_collate(p, CANON))
    o = oracle.canonicalize(p)
    assert_keys_equal(on, o)
    assert_keys_equal(off, o)
    scale = abs_scale(oracle, p)
    assert_values_close(on, o, scale)
    assert_values_close(off, o, scale)
    if n <= 50000 and nq >= 8:  # short segments: both paths fold in the reference's order
        assert bit_identical(on, o)
        assert bit_identical(off, o)


@pytest.mark.parametrize("cutoff", [1e-3, 0.5, 2.0])
def test_cutoff(cuda, oracle, cutoff):
    p = random_sum(40000, 1, 11, 10, "normal")
    on, off = both(lambda: gpu_collate(p, CANON, cutoff=cutoff))
    o = oracle.cutoff(oracle.canonicalize(p), cutoff)
    for g in (on, off):
        assert_keys_equal(g, o)
        assert_values_close(g, o, abs_scale(oracle, p))


def test_cancellation_and_phases(cuda, oracle):
    # every string with both phases and both signs; pairs that cancel exactly
    rng = np.random.default_rng(21)
    base = random_sum(3000, 1, 22, 9, "normal", flags="zero")
    _, first = np.unique(np.stack([base.x[0], base.z[0]]), axis=1, return_index=True)
    first = np.sort(first)  # distinct strings, so +v and -v meet alone
    bx, bz, bv = base.x[:, first], base.z[:, first], base.val[first]
    m = bv.shape[0]
    x = np.concatenate([bx] * 4, axis=1)
    z = np.concatenate([bz] * 4, axis=1)
    f = np.concatenate([np.full(m, k, np.uint8) for k in (0, 1, 2, 3)])
    v = np.concatenate([bv, rng.standard_normal(m), bv, rng.standard_normal(m)])
    p = Planes(x, z, f, v)  # flags 0 and 2 of one string cancel: +v and -(+v)
    on, off = both(lambda: gpu_collate(p, CANON))
    o = oracle.canonicalize(p)
    assert_keys_equal(on, o)
    assert bit_identical(on, o)
    assert bit_identical(off, o)
    assert set(np.unique(on.flags)) <= {1}  # phase-0 terms all cancelled


@pytest.mark.parametrize("terms", [128, 1024])
def test_product_workload(cuda, oracle, terms):
    a, b = W.product_operands(seed=terms + 1, terms=terms)
    a, b = as_planes(a), as_planes(b)
    on, off = both(lambda: gpu_multiply_collate(a, b))
    prod = oracle.multiply(a, b)
    o = oracle.canonicalize(prod)
    assert_keys_equal(on, o)
    assert_values_close(on, o, abs_scale(oracle, prod))
    assert_keys_equal(on, off)


def test_product_full_size(cuda):
    # the 4096 x 4096 product of the benchmark: 40 x / z bits + 24 index
    # bits, exactly one word.  Both paths against each other (the general
    # path is checked against the oracle at smaller sizes), and the
    # size-independent properties: sorted, unique, no zero coefficient.
    a, b = W.product_operands(seed=0, terms=4096)
    a, b = as_planes(a), as_planes(b)
    on, off = both(lambda: gpu_multiply_collate(a, b))
    assert on.n == off.n and on.n > 0
    assert_keys_equal(on, off)
    scale = np.abs(a.val).max() * np.abs(b.val).max() * 4096
    d = np.abs(on.val - off.val)
    assert float(d.max()) <= 1e-12 * scale
    assert np.all(on.val != 0.0)
    keys = np.stack([on.x[0], on.z[0], on.flags.astype(np.uint64)])
    order = np.lexsort(keys[::-1])
    assert np.array_equal(order, np.arange(on.n))
    same = (np.diff(on.x[0].astype(np.int64)) == 0) & (np.diff(on.z[0].astype(np.int64)) == 0) \
        & (np.diff(on.flags.astype(np.int64)) == 0)
    assert not same.any()


@contextlib.contextmanager
def tuned(key, value):
    L = _abi.lib()
    old = ctypes.c_int64()
    _abi.check(L.pl_get_tuning(key, ctypes.byref(old)), "pl_get_tuning")
    _abi.check(L.pl_set_tuning(key, value), "pl_set_tuning")
    try:
        yield
    finally:
        _abi.check(L.pl_set_tuning(key, old.value), "pl_set_tuning")


def _bits_equal(a, b):
    return (a.n == b.n and np.array_equal(a.x, b.x) and np.array_equal(a.z, b.z)
            and np.array_equal(a.flags, b.flags)
            and np.array_equal(a.val.view(np.uint64), b.val.view(np.uint64)))


@pytest.mark.parametrize("items", [8, 12, 16])
@pytest.mark.parametrize("n,nq,seed", [(1, 3, 31), (2, 4, 32), (3, 5, 33), (2049, 10, 34),
                                       (4097, 12, 35), (12289, 12, 36), (300001, 12, 37)])
@pytest.mark.parametrize("ahead", [0, 1, 7])
def test_l2_prefetch_digit_pass(cuda, oracle, items, n, nq, seed, ahead):
    # Digit passes that prefetch the tile `ahead` places on into L2 (0: one
    # wave) against passes without prefetch: bit-identical results, down to
    # one-key and odd-length final tiles (never prefetched: only whole tiles
    # are).
    p = random_sum(n, 1, seed, nq, "normal")
    with tuned(_abi.PL_TUNE_RADIX_ITEMS, items):
        with tuned(_abi.PL_TUNE_RADIX_PREFETCH, ahead):
            on = gpu_collate(p, CANON)
        with tuned(_abi.PL_TUNE_RADIX_PREFETCH, -1):
            off = gpu_collate(p, CANON)
    assert _bits_equal(on, off)
    o = oracle.canonicalize(p)
    assert_keys_equal(on, o)
    assert_values_close(on, o, abs_scale(oracle, p))


@pytest.mark.parametrize("items", [8, 16])
def test_l2_prefetch_digit_pass_product(cuda, items):
    # the 4096 x 4096 product of the benchmark with and without the prefetch
    a, b = W.product_operands(seed=0, terms=4096)
    a, b = as_planes(a), as_planes(b)
    with tuned(_abi.PL_TUNE_RADIX_ITEMS, items):
        with tuned(_abi.PL_TUNE_RADIX_PREFETCH, 0):
            on = gpu_multiply_collate(a, b)
        with tuned(_abi.PL_TUNE_RADIX_PREFETCH, -1):
            off = gpu_multiply_collate(a, b)
    assert on.n > 0 and _bits_equal(on, off)


@pytest.mark.parametrize("window", [2, 8, 16])
@pytest.mark.parametrize("n,nq,seed", [(3, 5, 51), (4097, 12, 52), (300001, 12, 53)])
def test_lookback_window(cuda, window, n, nq, seed):
    # every look-back window gives the same result as the default of 4
    p = random_sum(n, 1, seed, nq, "normal")
    with tuned(_abi.PL_TUNE_RADIX_WINDOW, window):
        on = gpu_collate(p, CANON)
        again = gpu_collate(p, CANON)
    off = gpu_collate(p, CANON)
    assert _bits_equal(on, off) and _bits_equal(on, again)


@pytest.mark.parametrize("items", [12, 16])
@pytest.mark.parametrize("terms,seed", [(4096, 0), (1024, 5), (2048, 7)])
def test_ten_bit_digits_product(cuda, oracle, items, terms, seed):
    # A product's index-packed keys sorted with 10-bit digits (1024 buckets,
    # 4 passes for 40 varying bits instead of 5) against 8-bit digits:
    # bit-identical; the smaller cases also against the oracle.
    a, b = W.product_operands(seed=seed, terms=terms)
    a, b = as_planes(a), as_planes(b)
    with tuned(_abi.PL_TUNE_RADIX_ITEMS, items):
        with tuned(_abi.PL_TUNE_RADIX_WIDE, 1):
            on = gpu_multiply_collate(a, b)
            again = gpu_multiply_collate(a, b)
        with tuned(_abi.PL_TUNE_RADIX_WIDE, -1):
            off = gpu_multiply_collate(a, b)
    assert on.n > 0 and _bits_equal(on, off) and _bits_equal(on, again)
    if terms <= 1024:
        prod = oracle.multiply(a, b)
        o = oracle.canonicalize(prod)
        assert_keys_equal(on, o)
        assert_values_close(on, o, abs_scale(oracle, prod))


@pytest.mark.parametrize("window", [2, 4, 8])
def test_ten_bit_digits_lookback_window(cuda, window):
    a, b = W.product_operands(seed=3, terms=2048)
    a, b = as_planes(a), as_planes(b)
    with tuned(_abi.PL_TUNE_RADIX_ITEMS, 12), tuned(_abi.PL_TUNE_RADIX_WINDOW, window):
        with tuned(_abi.PL_TUNE_RADIX_WIDE, 1):
            on = gpu_multiply_collate(a, b)
        with tuned(_abi.PL_TUNE_RADIX_WIDE, -1):
            off = gpu_multiply_collate(a, b)
    assert _bits_equal(on, off)


@pytest.mark.parametrize("backoff", [1, 4, 1024])
def test_lookback_backoff(cuda, backoff):
    # how soon a waiting tile backs off changes nothing in the result
    a, b = W.product_operands(seed=9, terms=2048)
    a, b = as_planes(a), as_planes(b)
    with tuned(_abi.PL_TUNE_RADIX_BACKOFF, backoff):
        on = gpu_multiply_collate(a, b)
    off = gpu_multiply_collate(a, b)
    assert _bits_equal(on, off)


@pytest.mark.parametrize("items", [8, 12, 16])
@pytest.mark.parametrize("terms,seed", [(4096, 0), (1024, 5), (96, 2)])
def test_fold_gathers_coefficients(cuda, oracle, items, terms, seed):
    # The fold taking each product's phase and coefficient from the operands
    # by index (the last digit pass moving keys only) against the last pass
    # gathering them: bit-identical; the smaller cases also against the oracle.
    a, b = W.product_operands(seed=seed, terms=terms)
    a, b = as_planes(a), as_planes(b)
    with tuned(_abi.PL_TUNE_RADIX_ITEMS, items):
        with tuned(_abi.PL_TUNE_FOLD_GATHER, 1):
            on = gpu_multiply_collate(a, b)
            again = gpu_multiply_collate(a, b)
        with tuned(_abi.PL_TUNE_FOLD_GATHER, -1):
            off = gpu_multiply_collate(a, b)
    assert on.n > 0 and _bits_equal(on, off) and _bits_equal(on, again)
    if terms <= 1024:
        prod = oracle.multiply(a, b)
        o = oracle.canonicalize(prod)
        assert_keys_equal(on, o)
        assert_values_close(on, o, abs_scale(oracle, prod))


def test_fold_gathers_with_cutoff(cuda, oracle):
    a, b = W.product_operands(seed=13, terms=512)
    a, b = as_planes(a), as_planes(b)
    with tuned(_abi.PL_TUNE_FOLD_GATHER, 1):
        on = gpu_multiply_collate(a, b, cutoff=0.05)
    with tuned(_abi.PL_TUNE_FOLD_GATHER, -1):
        off = gpu_multiply_collate(a, b, cutoff=0.05)
    assert _bits_equal(on, off)
