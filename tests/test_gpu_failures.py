"""Failure handling on a live device, with every failure made on the host
or by a bounded wait -- nothing here faults, traps or hangs the GPU.

* a cross-CTA wait on a flag that nothing sets gives up after the spin
  limit (PL_TUNE_SPIN_LIMIT) and reports PL_ERR_TIMEOUT; the context stays
  usable;
* an injected allocation failure (PL_TUNE_FAIL_ALLOC, a fake of the failing
  cudaMallocAsync) surfaces as PL_ERR_OOM and the state is reusable;
* a cancel flag stops a propagation between gates (PL_ERR_CANCELLED);
* the serving loop refuses a job whose fresh state alone exceeds the HBM
  budget, skips a cancelled job, and defers admission while a job's reserve
  does not fit beside the running job -- the other jobs' results unchanged.
"""
import ctypes as C
import threading

import numpy as np
import pytest

from paulib_b200 import _abi
from paulib_b200 import batch as B
from paulib_b200 import propagation as PR
from paulib_b200 import workloads as W
from paulib_b200.planes import Planes

pytestmark = pytest.mark.gpu


def _tune(key, value):
    _abi.check(_abi.lib().pl_set_tuning(key, value), "pl_set_tuning")


def test_bounded_wait_times_out_and_context_survives(cuda, oracle):
    L = _abi.lib()
    st = C.c_int(-1)
    try:
        _tune(_abi.PL_TUNE_SPIN_LIMIT, 64)
        _abi.check(L.pl_check_bounded_wait(C.byref(st)), "pl_check_bounded_wait")
        assert st.value == _abi.PL_ERR_TIMEOUT
    finally:
        _tune(_abi.PL_TUNE_SPIN_LIMIT, 0)
    # the default limit also ends (well under a second)
    st.value = -1
    _abi.check(L.pl_check_bounded_wait(C.byref(st)), "pl_check_bounded_wait")
    assert st.value == _abi.PL_ERR_TIMEOUT
    # and the device still computes correctly
    from gpu_util import gpu_multiply_collate
    from helpers import assert_keys_equal
    a, b = W.product_operands(seed=4, terms=200)
    a, b = Planes(a.x, a.z, a.flags, a.val), Planes(b.x, b.z, b.flags, b.val)
    assert_keys_equal(gpu_multiply_collate(a, b), oracle.canonicalize(oracle.multiply(a, b)))


def test_injected_allocation_failure_reports_oom(cuda, oracle):
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=24, layers=3)
    r = circ.rotations
    kw = dict(max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    with PR.State(1, 64) as st:  # must grow while propagating
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        _tune(_abi.PL_TUNE_FAIL_ALLOC, 1)
        try:
            with pytest.raises(_abi.PLError) as e:
                st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
            assert e.value.status == _abi.PL_ERR_OOM
        finally:
            _tune(_abi.PL_TUNE_FAIL_ALLOC, 0)
        # the same state runs the job again, correctly
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        g = Planes(*st.download())
    o = oracle.propagate(Planes(obs.x, obs.z, obs.flags, obs.val), Planes(r.x, r.z, r.flags, r.val),
                         circ.ops, **kw)
    assert g.n == o.n and np.array_equal(g.val.view(np.uint64), o.val.view(np.uint64))


def test_cancel_flag_stops_propagation_between_gates(cuda):
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=64, layers=20)
    r = circ.rotations
    kw = dict(max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    flag = np.zeros(1, np.int32)
    with PR.State(1, 1 << 20) as st:
        st.set_cancel_flag(flag)
        # set before the call: nothing runs, the observable stays
        flag[0] = 1
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        with pytest.raises(_abi.PLError) as e:
            st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        assert e.value.status == _abi.PL_ERR_CANCELLED
        assert st.size() == obs.n
        # set from another thread 40 ms into a ~0.3 s propagation
        flag[0] = 0
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        t = threading.Timer(0.04, lambda: flag.__setitem__(0, 1))
        t.start()
        with pytest.raises(_abi.PLError) as e:
            st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        t.join()
        assert e.value.status == _abi.PL_ERR_CANCELLED
        # cleared: the state propagates to the full result again
        st.set_cancel_flag(None)
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, **kw)
        assert st.size() == 1183321  # tests/golden/propagation_fixtures.json


def _small_jobs(count, seed):
    return W.batch_instances(seed=seed, count=count, qubit_choices=(16, 32), depth_range=(2, 3))


def _alone(inst):
    obs, circ = inst.observable, inst.circuit
    with PR.State(obs.x.shape[0]) as st:
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        r = circ.rotations
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, inst.max_weight, inst.cutoff)
        return st.zero_state_expectation()


def test_serve_rejects_oversized_and_skips_cancelled(cuda):
    jobs = _small_jobs(5, seed=31)
    # job 1: an observable of 2^21 terms -- its fresh state (5 buffers of
    # 25 B per term) alone is above the 128 MB budget
    n = 1 << 21
    rng = np.random.default_rng(0)
    big = W.SoA(rng.integers(0, 1 << 16, size=(1, n), dtype=np.uint64),
                rng.integers(0, 1 << 16, size=(1, n), dtype=np.uint64),
                np.zeros(n, np.uint8), rng.standard_normal(n), 16)
    jobs[1] = W.Instance(big, jobs[1].circuit, jobs[1].max_weight, jobs[1].cutoff)
    arr = np.linspace(0.0, 0.02, len(jobs))
    js = B.JobSet(jobs, arr)
    js.cancel[3] = 1
    r = B.serve(js, arr, lanes=2, hbm_budget=128 << 20, check=False)
    assert r.status[1] == _abi.PL_ERR_OOM
    assert r.status[3] == _abi.PL_ERR_CANCELLED
    assert r.rejected == 1
    for i in (0, 2, 4):
        assert r.status[i] == _abi.PL_OK
        assert r.expectation[i] == _alone(jobs[i]), i


def test_admission_defers_until_the_reserve_fits(cuda):
    # budget 1.5x a fresh state: the second job's reserve cannot sit beside
    # the first job's, so it is admitted only once the first has left
    jobs = _small_jobs(2, seed=41)
    js = B.JobSet(jobs)
    fresh = 5 * 25 * (1 << 16)
    r = B.batch_propagate(js, lanes=2, order="given", hbm_budget=int(1.5 * fresh))
    assert (r.status == 0).all()
    assert r.admission_waits >= 1
    first, second = np.argsort(r.start_s)
    assert r.start_s[second] >= r.end_s[first]
    for i, inst in enumerate(jobs):
        assert r.expectation[i] == _alone(inst), i
