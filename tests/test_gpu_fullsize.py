"""Parity at the full sizes the benchmarks time, through the C ABI.

* product + canonicalize, 4096 x 4096 (16.8M products, the headline step):
  against the reference build (oracle/_ref) run at test time -- strings,
  phases and order exact; coefficients within 1e-12 of the summed
  magnitudes of each key's contributions (the reference's own build
  reassociates its segment sums under -ffast-math, and long segments are
  summed by a fixed tree here).
* commutator 16384 x 16384 at 256 qubits (2.7e8 pairs), then canonicalize +
  cutoff(1e-14): the raw commutator output against the reference's
  single-threaded commutator (the one deterministic CPU order,
  PauliSumOperations.h:316-346) bit for bit, then the collated sum as above.
* Heisenberg propagation, 64 qubits x 20 layers (peak ~8M terms), and
  sampled jobs of the mixed batch: the final sums' SHA-256 digests, term
  counts and zero_state_expectation against fixtures that
  tests/golden/make_fixtures.py made with the reference build (propagated
  sums are bit-identical to the reference; expectations within 1e-10).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from gpu_util import as_planes, gpu_collate, gpu_commutator, gpu_multiply_collate
from helpers import assert_keys_equal, assert_values_close_sorted, bit_identical
from paulib_b200 import propagation as PR
from paulib_b200 import workloads as W
from paulib_b200.planes import Planes

pytestmark = pytest.mark.gpu

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "propagation_fixtures.json")


def _fixtures():
    with open(FIXTURES) as fh:
        return json.load(fh)


def _digest(p: Planes) -> str:
    h = hashlib.sha256()
    for a, dt in ((p.x, np.uint64), (p.z, np.uint64), (p.flags, np.uint8), (p.val, np.float64)):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


def _abs_scale(reference, raw: Planes) -> Planes:
    """Per canonical key (x, z, phase): the sum of |contributions|."""
    return reference.sort_and_combine(Planes(raw.x, raw.z, raw.flags & np.uint8(1),
                                             np.abs(raw.val)))


def test_product_collate_4096x4096_vs_reference(cuda, reference):
    a, b = W.product_operands(seed=1)  # the operands bench.py times
    a, b = as_planes(a), as_planes(b)
    g = gpu_multiply_collate(a, b)
    prod = reference.multiply(a, b)
    ref = reference.canonicalize(prod)
    assert g.n == ref.n > 3_000_000
    assert_keys_equal(g, ref)
    assert_values_close_sorted(g, ref, _abs_scale(reference, prod))


def test_commutator_16384x16384_as4_vs_reference(cuda, reference):
    a, b = W.window_sums(seed=3)  # the operands of the commutator benchmark
    a, b = as_planes(a), as_planes(b)
    raw_g = gpu_commutator(a, b, capacity=a.n * b.n // 64)
    threads = reference.threads
    reference.set_threads(1)  # the deterministic (lhs-major) CPU emission order
    try:
        raw = reference.commutator(a, b)
    finally:
        reference.set_threads(threads)
    assert raw_g.n == raw.n > 3_000_000
    assert_keys_equal(raw_g, raw)
    assert bit_identical(raw_g, raw)
    g = gpu_collate(raw_g, cutoff=1e-14)
    ref = reference.cutoff(reference.canonicalize(raw), 1e-14)
    assert g.n == ref.n > 1_000_000
    assert_keys_equal(g, ref)
    assert_values_close_sorted(g, ref, _abs_scale(reference, raw))


def _propagate(obs, circ, max_weight, cutoff):
    with PR.State(obs.array_size, 1 << 20) as st:
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, max_weight, cutoff)
        g = Planes(*st.download())
        e = st.zero_state_expectation()
    return g, e


def _check_fixture(name, obs, circ, max_weight, cutoff):
    fx = _fixtures()[name]
    assert (fx["num_qubits"], fx["rotations"]) == (circ.num_qubits, circ.n_rotations)
    g, e = _propagate(obs, circ, max_weight, cutoff)
    assert g.n == fx["terms"]
    assert _digest(g) == fx["sha256"], "final sum differs from the reference's"
    assert abs(e - fx["expectation"]) <= 1e-10


def test_heisenberg_64q_20_layers_vs_reference_fixture(cuda):
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=64, layers=20)
    _check_fixture("heisenberg_64q_20l", obs, circ, tr["max_weight"], tr["cutoff"])


def _batch_fixture_jobs():
    names = sorted(k for k in _fixtures() if k.startswith("batch_job_"))
    return [int(k.rsplit("_", 1)[1]) for k in names]


@pytest.mark.parametrize("index", _batch_fixture_jobs())
def test_batch_job_vs_reference_fixture(cuda, index):
    j = W.batch_instances()[index]
    _check_fixture(f"batch_job_{index}", j.observable, j.circuit, j.max_weight, j.cutoff)


def test_heavy_job_first_10_layers_vs_reference_fixture(cuda):
    from paulib_b200.benchmarks import sub_circuit
    h = W.heavy_instance()
    _check_fixture("heavy_first10", h.observable, sub_circuit(h.circuit, 10), h.max_weight,
                   h.cutoff)


def test_batch_executor_matches_fixtures(cuda):
    # the same sampled jobs through the multi-lane executor, all at once
    from paulib_b200 import batch as B
    fx = _fixtures()
    idx = _batch_fixture_jobs()
    jobs = W.batch_instances()
    r = B.batch_propagate([jobs[i] for i in idx], lanes=4)
    for k, i in enumerate(idx):
        assert r.final_terms[k] == fx[f"batch_job_{i}"]["terms"]
        assert abs(r.expectation[k] - fx[f"batch_job_{i}"]["expectation"]) <= 1e-10
