"""Host-side logic of the batch and serving forms, without a GPU: argument
validation in the C ABI (before any device work), the job table built for
it, and the Poisson arrival stream."""
import ctypes as C

import numpy as np

from paulib_b200 import _abi
from paulib_b200 import batch as B
from paulib_b200 import workloads as W


def _call(fn, js, opts):
    res = (_abi.JobResult * max(len(js), 1))()
    st = _abi.BatchStats()
    return fn(js.jobs, len(js), C.byref(opts), res, C.byref(st))


def test_invalid_options_rejected_before_device_work():
    lib = _abi.lib()
    js = B.JobSet(W.batch_instances(count=2, depth_range=(1, 1)))
    bad = B._opts(0, True, "longest", 0, 0)
    assert _call(lib.pl_batch_propagate, js, bad) == _abi.PL_ERR_INVALID_ARG
    ok = B._opts(2, True, "longest", 0, 0)
    js.jobs[1].array_size = 0
    assert _call(lib.pl_batch_propagate, js, ok) == _abi.PL_ERR_INVALID_ARG
    js.jobs[1].array_size = 1
    js.jobs[0].arrival_s = -1.0
    assert _call(lib.pl_serve, js, ok) == _abi.PL_ERR_INVALID_ARG


def test_jobset_fields():
    insts = W.batch_instances(count=3, depth_range=(2, 3))
    js = B.JobSet(insts, arrivals=[0.0, 0.5, 1.5])
    for i, inst in enumerate(insts):
        j = js.jobs[i]
        assert j.array_size == inst.observable.x.shape[0]
        assert j.n_rot == inst.circuit.rotations.val.shape[0]
        assert j.n_ops == inst.circuit.ops.shape[0]
        assert j.trunc.max_weight == inst.max_weight
        assert j.trunc.coefficient_cutoff == inst.cutoff
    assert js.jobs[2].arrival_s == 1.5


def test_poisson_arrivals():
    a = B.poisson_arrivals(20000, rate_per_s=50.0, seed=1)
    assert np.all(np.diff(a) > 0)
    assert abs(a[-1] / len(a) - 1 / 50.0) < 0.05 / 50.0 * 10
    assert np.array_equal(a, B.poisson_arrivals(20000, rate_per_s=50.0, seed=1))
