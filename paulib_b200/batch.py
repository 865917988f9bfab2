"""Many propagations on one device: batch and serving (pl_batch_propagate /
pl_serve), the form of propagate_expectation (PauliPropagation.h:65-71)
that keeps several device-resident Pauli sums in flight at once.

A job is one workloads.Instance (observable, circuit, truncation).  The
executor runs jobs on ``lanes`` device states, each with its own stream and
host thread, replays runs of single-qubit rotations from captured CUDA
graphs, admits work against an HBM budget and returns per-job results and
timestamps.  A job's result does not depend on what runs beside it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi

U64_MAX = (1 << 64) - 1


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


class JobSet:
    """ctypes job array over workloads.Instance objects (arrays kept alive).

    ``cancel`` is an int32 array, one flag per job: setting flag i to a
    non-zero value (from any host thread, at any time) makes job i stop
    between gates -- or not start -- with PL_ERR_CANCELLED."""

    def __init__(self, instances, arrivals=None):
        self.instances = list(instances)
        self._keep = []
        self.cancel = np.zeros(max(len(self.instances), 1), np.int32)
        self.jobs = (_abi.Job * max(len(self.instances), 1))()
        for i, inst in enumerate(self.instances):
            obs, circ = inst.observable, inst.circuit
            r = circ.rotations
            aw = int(obs.x.shape[0])
            arrs = [np.ascontiguousarray(obs.x, np.uint64), np.ascontiguousarray(obs.z, np.uint64),
                    np.ascontiguousarray(obs.flags, np.uint8),
                    np.ascontiguousarray(obs.val, np.float64),
                    np.ascontiguousarray(r.x, np.uint64).reshape(aw, -1),
                    np.ascontiguousarray(r.z, np.uint64).reshape(aw, -1),
                    np.ascontiguousarray(r.flags, np.uint8),
                    np.ascontiguousarray(r.val, np.float64),
                    np.ascontiguousarray(circ.ops, np.int32).reshape(-1, 3)]
            self._keep.append(arrs)
            j = self.jobs[i]
            j.array_size = aw
            j.obs_x, j.obs_z, j.obs_flags, j.obs_val = (_p(a) for a in arrs[:4])
            j.obs_n = arrs[3].shape[0]
            j.rot_x, j.rot_z, j.rot_flags, j.rot_theta = (_p(a) for a in arrs[4:8])
            j.n_rot = arrs[7].shape[0]
            j.ops = _p(arrs[8])
            j.n_ops = arrs[8].shape[0]
            j.trunc.max_weight = U64_MAX if inst.max_weight is None else int(inst.max_weight)
            j.trunc.coefficient_cutoff = float(inst.cutoff or 0.0)
            j.trunc.max_terms = U64_MAX
            j.arrival_s = 0.0 if arrivals is None else float(arrivals[i])
            j.cancel = self.cancel[i:].ctypes.data_as(C.c_void_p)

    def estimate(self, i: int):
        """(terms, bytes) admission estimate of job i (pl_job_estimate)."""
        t, b = C.c_uint64(), C.c_uint64()
        _abi.check(_abi.lib().pl_job_estimate(C.byref(self.jobs[i]), C.byref(t), C.byref(b)),
                   "pl_job_estimate")
        return t.value, b.value

    def __len__(self):
        return len(self.instances)


@dataclass
class BatchResult:
    expectation: np.ndarray
    final_terms: np.ndarray
    status: np.ndarray
    lane: np.ndarray
    start_s: np.ndarray
    end_s: np.ndarray
    wall_s: float
    peak_bytes: int
    budget_waits: int
    rejected: int = 0
    admission_waits: int = 0


def _opts(lanes, graphs, order, hbm_budget, keep_bytes):
    o = _abi.BatchOpts()
    o.lanes = int(lanes)
    o.use_graphs = 1 if graphs else 0
    o.order = _abi.PL_ORDER_LONGEST_FIRST if order == "longest" else _abi.PL_ORDER_GIVEN
    o.hbm_budget = int(hbm_budget or 0)
    o.keep_bytes = int(keep_bytes or 0)
    o.sync_stream = None
    return o


def _collect(res, n, st) -> BatchResult:
    g = lambda f, dt: np.array([getattr(res[i], f) for i in range(n)], dt)
    return BatchResult(g("expectation", np.float64), g("final_terms", np.int64),
                       g("status", np.int32), g("lane", np.int32), g("start_s", np.float64),
                       g("end_s", np.float64), st.wall_s, st.peak_bytes, st.budget_waits,
                       st.jobs_rejected, st.admission_waits)


def _run(fn, js: JobSet, opts, check: bool) -> BatchResult:
    n = len(js)
    res = (_abi.JobResult * max(n, 1))()
    st = _abi.BatchStats()
    rc = fn(js.jobs, n, C.byref(opts), res, C.byref(st))
    out = _collect(res, n, st)
    if check:
        _abi.check(rc, fn.__name__)
    return out


def batch_propagate(jobs, lanes=8, graphs=True, order="longest", hbm_budget=0, keep_bytes=0,
                    check=True) -> BatchResult:
    """Run every job (a JobSet or a list of workloads.Instance)."""
    js = jobs if isinstance(jobs, JobSet) else JobSet(jobs)
    return _run(_abi.lib().pl_batch_propagate, js, _opts(lanes, graphs, order, hbm_budget,
                                                          keep_bytes), check)


def serve(jobs, arrivals=None, lanes=8, graphs=True, hbm_budget=0, keep_bytes=0,
          check=True) -> BatchResult:
    """Serve jobs arriving at ``arrivals`` (seconds from the call's start)."""
    js = jobs if isinstance(jobs, JobSet) else JobSet(jobs, arrivals)
    return _run(_abi.lib().pl_serve, js, _opts(lanes, graphs, "given", hbm_budget, keep_bytes),
                check)


def plain(jobs, graphs=False) -> BatchResult:
    """The one-instance-at-a-time GPU path: one lane, jobs in the given order."""
    return batch_propagate(jobs, lanes=1, graphs=graphs, order="given")


def poisson_arrivals(count: int, rate_per_s: float, seed: int = 11) -> np.ndarray:
    """Arrival times of a Poisson process (exponential gaps), seeded."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / float(rate_per_s), size=count))


def latency_percentiles(r: BatchResult, arrivals) -> dict:
    lat = r.end_s - np.asarray(arrivals, np.float64)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
