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


def _light_cone_py(inst):
    """Light-cone support of the observable, restated for the check."""
    obs, circ = inst.observable, inst.circuit
    aw = obs.x.shape[0]
    sup = set()
    for k in range(aw):
        w = int(obs.x[k, 0]) | int(obs.z[k, 0])
        sup |= {64 * k + b for b in range(64) if (w >> b) & 1}
    for kind, a, b in circ.ops[::-1]:
        if kind == W.OP_CNOT and (a in sup or b in sup):
            sup |= {int(a), int(b)}
    return len(sup)


def test_job_estimate_bounds():
    # pl_job_estimate is host arithmetic: the Frobenius bound, the weight
    # bound over the light cone, and the byte model, restated here.
    from math import comb
    insts = W.batch_instances(seed=3, count=6, qubit_choices=(16, 64), depth_range=(1, 3))
    js = B.JobSet(insts)
    for i, inst in enumerate(insts):
        s = _light_cone_py(inst)
        w = inst.max_weight
        weight = 2 * sum(comb(s, k) * 3 ** k for k in range(min(w, s) + 1))
        fro = int(2 * float(np.abs(inst.observable.val).sum()) ** 2 / inst.cutoff ** 2)
        terms, nbytes = js.estimate(i)
        want = max(min(weight, fro), inst.observable.n)
        assert abs(terms - want) <= 1e-9 * want, (i, s, terms, want)
        S = 16 * inst.observable.x.shape[0] + 9
        assert abs(nbytes - (20 * S * terms + (64 << 20))) <= 1e-9 * nbytes
    # no cutoff: only the weight bound; no weight limit either: 2 * 4^s
    j = js.jobs[0]
    j.trunc.coefficient_cutoff = 0.0
    j.trunc.max_weight = (1 << 64) - 1
    t = C.c_uint64()
    b = C.c_uint64()
    assert _abi.lib().pl_job_estimate(C.byref(j), C.byref(t), C.byref(b)) == _abi.PL_OK
    s = _light_cone_py(insts[0])
    assert t.value == 2 * 4 ** s
