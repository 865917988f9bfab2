"""GPU parity of the per-pair and per-term kernels against the oracle,
through the C ABI: outer product (pl_multiply and the launch_gpu_mul_soa
drop-in), commutator (pl_commutator and the launch_gpu_commutator_soa
drop-in), apply_CNOT, zero_state_expectation.

Integer work must match bit for bit; products are single roundings, so the
coefficients must match bit for bit too.  The reference GPU tests compare
after sort_and_combine because its atomics scramble the order
(tests/GpuPauliSumTests.cpp:256-343); this implementation is ordered, so the
comparison here is term by term in the CPU order.
"""
import math

import numpy as np
import pytest

from gpu_util import (as_planes, gpu_cnot, gpu_commutator, gpu_multiply, gpu_zero_state)
from helpers import assert_keys_equal, bit_identical, planes, random_sum
from paulib_b200.planes import Planes
from paulib_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("row", "IXYZ")
def test_single_qubit_products(cuda, oracle, row):
    # GpuPauliSumTests.cpp:145-204: every single-qubit product and its flag.
    for col in "IXYZ":
        a, b = planes([(row, 2.5)]), planes([(col, -4.0)])
        g, o = gpu_multiply(a, b), oracle.multiply(a, b)
        assert_keys_equal(g, o)
        assert bit_identical(g, o)


@pytest.mark.parametrize("words,n,m", [(1, 13, 7), (2, 10, 10), (8, 30, 20), (8, 100, 100),
                                       (16, 9, 11), (3, 1, 257)])
@pytest.mark.parametrize("dropin", [False, True])
def test_multiply_random(cuda, oracle, words, n, m, dropin):
    # GpuPauliSumTests.cpp:256-300 (AS = 1, 2, 8 up to 100x100) and more.
    a, b = random_sum(n, words, 42 + n), random_sum(m, words, 99 + m, coeffs="normal")
    g, o = gpu_multiply(a, b, dropin=dropin), oracle.multiply(a, b)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_multiply_config_operands(cuda, oracle):
    a, b = W.product_operands(seed=1, terms=512)
    a, b = as_planes(a), as_planes(b)
    g, o = gpu_multiply(a, b), oracle.multiply(a, b)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


@pytest.mark.parametrize("mul_i", [False, True])
@pytest.mark.parametrize("dropin", [False, True])
def test_commutator_matches_cpu_order(cuda, oracle, mul_i, dropin):
    # GpuPauliSumTests.cpp:306-337 (200x150 over 40 qubits, i-commutator).
    a = random_sum(200, 1, 11, 40)
    b = random_sum(150, 1, 22, 40)
    a.val[:] = 0.5 + (np.arange(200) % 7)
    b.val[:] = np.where(np.arange(150) % 2, -1.0, 1.0) * (0.25 + np.arange(150) % 5)
    g, o = gpu_commutator(a, b, mul_i, dropin=dropin), oracle.commutator(a, b, mul_i)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


@pytest.mark.parametrize("terms", [300, 2000])
def test_commutator_windowed(cuda, oracle, terms):
    a, b = W.window_sums(seed=3, terms=terms)
    a, b = as_planes(a), as_planes(b)
    g, o = gpu_commutator(a, b), oracle.commutator(a, b)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


@pytest.mark.parametrize("n,m,words,nq", [(2500, 1777, 4, 256), (4099, 1031, 1, 40),
                                         (1024, 4096, 2, 100)])
@pytest.mark.parametrize("mul_i", [False, True])
def test_commutator_two_pass_form(cuda, oracle, n, m, words, nq, mul_i):
    # n * m >= 2^22 pairs take the bitmask form (k_comm_mask + k_comm_emit):
    # same terms, same order, same values as the single-threaded CPU
    # commutator; sizes not multiples of the tile shapes
    a = random_sum(n, words, 5 + n, nq, "normal")
    b = random_sum(m, words, 6 + m, nq, "normal")
    # random strings anticommute about half the time: room for every pair
    g, o = gpu_commutator(a, b, mul_i, capacity=n * m), oracle.commutator(a, b, mul_i)
    assert_keys_equal(g, o)
    assert bit_identical(g, o)


def test_commutator_two_pass_capacity(cuda, oracle):
    from paulib_b200 import _abi
    a, b = random_sum(2100, 1, 5, 20), random_sum(2100, 1, 6, 20)
    full = oracle.commutator(a, b)
    with pytest.raises(_abi.PLError) as e:
        gpu_commutator(a, b, capacity=full.n // 2)
    assert e.value.status == _abi.PL_ERR_CAPACITY


def test_commutator_commuting_inputs(cuda):
    # GpuPauliSumTests.cpp:339-343.
    g = gpu_commutator(planes([("ZI", 1.0)]), planes([("IZ", 1.0)]))
    assert g.n == 0


def test_commutator_capacity_reported(cuda, oracle):
    from paulib_b200 import _abi
    a, b = random_sum(64, 1, 5, 20), random_sum(64, 1, 6, 20)
    full = oracle.commutator(a, b)
    with pytest.raises(_abi.PLError) as e:
        gpu_commutator(a, b, capacity=max(full.n // 2, 1))
    assert e.value.status == _abi.PL_ERR_CAPACITY


def test_dropin_commutator_is_async_and_counts_overflow(cuda, oracle):
    # The drop-in launcher is asynchronous like the reference's
    # (paulib_gpu_api.h:35-42): no status read-back; an output that does not
    # fit shows as a final count above the capacity, and the slots that fit
    # hold the first terms in order.
    import torch
    from gpu_util import dev, host
    from paulib_b200 import _abi
    a, b = random_sum(64, 1, 5, 20), random_sum(64, 1, 6, 20)
    full = oracle.commutator(a, b)
    cap = max(full.n // 2, 1)
    da, db = dev(a), dev(b)
    out = _abi.DeviceSum(1, cap)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    L = _abi.lib()
    L.launch_gpu_commutator_soa(1, 0, *da.ptrs(), *db.ptrs(), *out.ptrs(), cnt.data_ptr(),
                                a.n, b.n, cap, _abi.stream_ptr())
    torch.cuda.synchronize()
    assert _abi.last_error() == _abi.PL_OK
    assert int(cnt.item()) == full.n > cap
    out.n = cap
    g = host(out)
    head = Planes(full.x[:, :cap], full.z[:, :cap], full.flags[:cap], full.val[:cap])
    assert_keys_equal(g, head)
    assert bit_identical(g, head)


@pytest.mark.parametrize("words,c,t", [(1, 0, 1), (1, 3, 9), (2, 0, 70), (2, 100, 5),
                                       (1, 63, 62)])
def test_cnot(cuda, oracle, words, c, t):
    p = random_sum(1000, words, 7 + c + t)
    g, o = gpu_cnot(p, c, t), oracle.apply_cnot(p, c, t)
    assert_keys_equal(g, o)
    assert np.array_equal(g.val, o.val)


def test_cnot_truth_table(cuda, oracle):
    from test_oracle_golden import CNOT
    from helpers import to_str
    for inp, out in CNOT.items():
        assert to_str(gpu_cnot(planes([(inp, 1.0)]), 0, 1), 2) == f"1.000000 * {out}\n"


@pytest.mark.parametrize("words,n", [(1, 0), (1, 5), (2, 100000), (4, 3333)])
def test_zero_state_expectation(cuda, oracle, words, n):
    p = random_sum(n, words, 3, coeffs="normal")
    # make a good fraction of terms X-free so the sum is non-trivial
    p.x[:, ::3] = 0
    g, o = gpu_zero_state(p), oracle.zero_state_expectation(p)
    scale = max(1.0, float(np.abs(p.val).sum()))
    assert abs(g - o) <= 1e-12 * scale
