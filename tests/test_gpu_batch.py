"""Batch and serving forms of propagate_expectation (pl_batch_propagate,
pl_serve) and graph-replayed rotation runs, against the plain path and the
oracle, through the C ABI.

A job's result may not depend on the mix it runs in: expectations and final
term counts must be bit-identical to the same job run alone on the plain
one-instance-at-a-time path (no graphs, one lane).
"""
import numpy as np
import pytest

from paulib_b200.planes import Planes
from paulib_b200 import batch as B
from paulib_b200 import propagation as PR
from paulib_b200 import workloads as W

pytestmark = pytest.mark.gpu


def light_instances(count=12, seed=21):
    # the batch workload's distribution at its shallow end (<= ~1e6 terms)
    return W.batch_instances(seed=seed, count=count, qubit_choices=(16, 32, 64, 128),
                             depth_range=(2, 4))


def alone(inst, graphs=False):
    obs, circ = inst.observable, inst.circuit
    with PR.State(obs.x.shape[0]) as st:
        st.use_graphs(graphs)
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, inst.max_weight, inst.cutoff)
        return st.zero_state_expectation(), st.download()


def test_graph_runs_match_plain(cuda):
    for inst in light_instances(4, seed=3):
        e0, s0 = alone(inst, graphs=False)
        e1, s1 = alone(inst, graphs=True)
        assert e0 == e1
        for a, b in zip(s0, s1):
            assert np.array_equal(a, b)


def test_graph_runs_match_oracle(cuda, oracle):
    inst = W.batch_instances(seed=5, count=1, qubit_choices=(16,), depth_range=(3, 3))[0]
    obs, circ = inst.observable, inst.circuit
    P = lambda s: Planes(s.x, s.z, s.flags, s.val)
    o = oracle.propagate(P(obs), P(circ.rotations), circ.ops, max_weight=inst.max_weight,
                         cutoff=inst.cutoff)
    e, (x, z, f, v) = alone(inst, graphs=True)
    assert np.array_equal(x, o.x) and np.array_equal(z, o.z) and np.array_equal(f, o.flags)
    assert np.array_equal(v.view(np.uint64), o.val.view(np.uint64))
    assert abs(e - oracle.zero_state_expectation(o)) <= 1e-10


@pytest.mark.parametrize("lanes,graphs", [(4, True), (3, False)])
def test_batch_same_alone_and_in_mix(cuda, lanes, graphs):
    insts = light_instances()
    r = B.batch_propagate(insts, lanes=lanes, graphs=graphs, order="longest")
    assert (r.status == 0).all()
    assert set(r.lane.tolist()) <= set(range(lanes))
    for i, inst in enumerate(insts):
        e, s = alone(inst)
        assert r.expectation[i] == e, i
        assert r.final_terms[i] == s[3].shape[0], i


def test_serve_same_alone_and_in_mix(cuda):
    insts = light_instances(10, seed=8)
    arr = B.poisson_arrivals(len(insts), rate_per_s=200.0, seed=2)
    r = B.serve(insts, arr, lanes=4, graphs=True)
    assert (r.status == 0).all()
    assert (r.start_s >= arr - 1e-6).all() and (r.end_s >= r.start_s).all()
    for i, inst in enumerate(insts):
        assert r.expectation[i] == alone(inst)[0], i
    lat = B.latency_percentiles(r, arr)
    assert 0.0 <= lat["p50_s"] <= lat["p99_s"]


def test_small_budget_still_correct(cuda):
    # a budget below what four lanes would like to hold: lanes wait for and
    # give back memory, results unchanged
    insts = light_instances(8, seed=13)
    r = B.batch_propagate(insts, lanes=4, graphs=True, hbm_budget=256 << 20,
                          keep_bytes=64 << 20)
    assert (r.status == 0).all()
    for i, inst in enumerate(insts):
        assert r.expectation[i] == alone(inst)[0], i
