#!/usr/bin/env python
"""Generate the full-size propagation fixtures with the reference build.

TEST INFRASTRUCTURE: runs the reference's own header-only implementation
(``oracle/_ref``, built by ``oracle/Makefile``) on the seeded propagation
workloads whose CPU run takes minutes, and records for each one the final
term count, a SHA-256 digest of the final SoA planes (x, z, flags, value
bytes in the final term order) and ``zero_state_expectation``.  The GPU
tests (``tests/test_gpu_fullsize.py``) recompute the same workloads through
the C ABI and compare: propagated sums are bit-identical to the reference
(every canonical key receives at most one old and one new contribution per
rotation), so the digests must match exactly.

    python tests/golden/make_fixtures.py [--only NAME ...] [--threads T]

Workloads (``paulib_b200.workloads``):
  heisenberg_64q_20l   sum_i Z_i on 64 qubits, 20 brickwork layers,
                       cutoff 1e-4, max weight 8 (PauliPropagation.h:54-71)
  batch_job_<i>        jobs of the 512-job mixed batch (seed 4): one each of
                       16, 32, 64 and 128 qubits, the cheapest few by depth
  heavy_first10        the first 10 brickwork layers of the heavy serving
                       job (128 qubits), cutoff 1e-5, max weight 10
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Planes, Reference  # noqa: E402
from paulib_b200 import workloads as W  # noqa: E402
from paulib_b200.benchmarks import sub_circuit  # noqa: E402

OUT = os.path.join(HERE, "propagation_fixtures.json")


def planes_digest(x, z, flags, val) -> str:
    h = hashlib.sha256()
    for a, dt in ((x, np.uint64), (z, np.uint64), (flags, np.uint8), (val, np.float64)):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


def batch_picks(jobs):
    """Jobs of the mixed batch checked at full size: per qubit count, the
    shallowest job (lowest index among equals), and a second, deeper
    16-qubit job."""
    picks = []
    for nq in (16, 32, 64, 128):
        cand = [(j.circuit.meta["layers"], i) for i, j in enumerate(jobs)
                if j.circuit.num_qubits == nq]
        picks.append(min(cand)[1])
    deep16 = [(-j.circuit.meta["layers"], i) for i, j in enumerate(jobs)
              if j.circuit.num_qubits == 16]
    picks.append(min(deep16)[1])
    return picks


def workloads():
    """name -> (observable, circuit, max_weight, cutoff)"""
    out = {}
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=64, layers=20)
    out["heisenberg_64q_20l"] = (obs, circ, tr["max_weight"], tr["cutoff"])
    jobs = W.batch_instances()
    for i in batch_picks(jobs):
        j = jobs[i]
        out[f"batch_job_{i}"] = (j.observable, j.circuit, j.max_weight, j.cutoff)
    h = W.heavy_instance()
    out["heavy_first10"] = (h.observable, sub_circuit(h.circuit, 10), h.max_weight, h.cutoff)
    return out


def as_planes(s) -> Planes:
    return Planes(s.x, s.z, s.flags, s.val)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    a = ap.parse_args(argv)
    R = Reference(threads=a.threads)
    try:
        with open(OUT) as fh:
            data = json.load(fh)
    except (OSError, ValueError):
        data = {}
    for name, (obs, circ, mw, cut) in workloads().items():
        if a.only and name not in a.only:
            continue
        t0 = time.perf_counter()
        res = R.propagate(as_planes(obs), as_planes(circ.rotations), circ.ops,
                          max_weight=mw, cutoff=cut)
        dt = time.perf_counter() - t0
        data[name] = {
            "num_qubits": int(circ.num_qubits), "layers": int(circ.meta["layers"]),
            "rotations": int(circ.n_rotations), "max_weight": int(mw), "cutoff": float(cut),
            "terms": int(res.n), "sha256": planes_digest(res.x, res.z, res.flags, res.val),
            "expectation": float(R.zero_state_expectation(res)),
            "generator": f"{os.path.basename(R.path)}, {R.threads} threads, {dt:.1f} s",
        }
        print(name, data[name], flush=True)
        with open(OUT, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
            fh.write("\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
