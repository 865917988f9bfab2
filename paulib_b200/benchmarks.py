"""Secondary benchmark workloads for bench.py (--workload ...).

propagation  Heisenberg propagation of sum_i Z_i through a 64-qubit, 20-layer
             brickwork CNOT+RX+RZ circuit, cutoff 1e-4, max weight 8, then
             zero_state_expectation (metric: propagations/s).
commutator   [A, B] of two PauliSum<256,double> of 16384 windowed terms,
             then canonicalize + cutoff(1e-14) (metric: pairs collated/s).
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _abi
from . import propagation as PR
from . import workloads as W


def _sync():
    import torch
    torch.cuda.synchronize()


def run(name, args, rank, local, ws):
    import torch
    torch.cuda.set_device(local)
    if name == "propagation":
        return _propagation(args, rank, ws)
    if name == "commutator":
        return _commutator(args, rank, ws)
    raise ValueError(name)


def _propagation(args, rank, ws):
    import torch
    obs, circ, tr = W.heisenberg_workload(seed=2 + rank, num_qubits=64, layers=20)
    r = circ.rotations
    st = PR.State(1, 1 << 24)

    def once():
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, tr["max_weight"], tr["cutoff"])
        return st.zero_state_expectation()

    steps = max(1, min(args.steps, 5))
    for _ in range(max(1, min(args.warmup, 2))):
        e = once()
    _abi.profile_reset(False)
    _sync()
    times = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        e = once()
        e1.record()
        _sync()
        times.append(e0.elapsed_time(e1))
    launches, _, _, _ = _abi.profile_read()
    final = st.size()
    ms = sum(times) / steps
    return {"metric": "propagations/s", "value": ws * 1e3 / ms, "unit": "propagations/s",
            "n_gpus": ws, "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 keys / f64 coefficients", "data": "synthetic, seeded",
            "config": {"workload": "propagation: sum_i Z_i, 64 qubits, 20 brickwork layers "
                                   "CNOT+RX+RZ, cutoff 1e-4, max_weight 8",
                       "rotations": int(r.n), "final_terms": final, "expectation": e},
            "gpu_launches": int(launches // steps)}


def _commutator(args, rank, ws):
    import torch
    a, b = W.window_sums(seed=3 + rank)
    L = _abi.lib()
    da = _abi.DeviceSum.from_host(a.x, a.z, a.flags, a.val)
    db = _abi.DeviceSum.from_host(b.x, b.z, b.flags, b.val)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    sp = _abi.stream_ptr()
    # sizing call: capacity 0 reports the emitted count
    rc = L.pl_commutator(4, 0, *da.ptrs(), a.n, *db.ptrs(), b.n, *da.ptrs(), 0,
                         cnt.data_ptr(), sp)
    assert rc in (_abi.PL_OK, _abi.PL_ERR_CAPACITY), rc
    emitted = int(cnt.item())
    out = _abi.DeviceSum(4, emitted)
    col = _abi.DeviceSum(4, emitted)
    nb = C.c_size_t()
    _abi.check(L.pl_collate_workspace_size(4, emitted, C.byref(nb)))
    wsb = _abi.workspace(nb.value)
    opts = _abi.CollateOpts(_abi.PL_COLLATE_CANONICALIZE, 0, 1e-14, _abi.UINT64_MAX)
    n_out = C.c_int64()

    def once():
        cnt.zero_()
        _abi.check(L.pl_commutator(4, 0, *da.ptrs(), a.n, *db.ptrs(), b.n, *out.ptrs(), emitted,
                                   cnt.data_ptr(), sp), "pl_commutator")
        _abi.check(L.pl_collate(4, *out.ptrs(), emitted, *col.ptrs(), emitted, C.byref(n_out),
                                C.byref(opts), wsb.data_ptr(), nb.value, sp), "pl_collate")
        return n_out.value

    for _ in range(args.warmup):
        once()
    _sync()
    _abi.profile_reset(True)
    t_comm, t_all = [], []
    steps = max(3, min(args.steps, 50))
    for _ in range(steps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        cnt.zero_()
        L.pl_commutator(4, 0, *da.ptrs(), a.n, *db.ptrs(), b.n, *out.ptrs(), emitted,
                        cnt.data_ptr(), sp)
        e1.record()
        L.pl_collate(4, *out.ptrs(), emitted, *col.ptrs(), emitted, C.byref(n_out),
                     C.byref(opts), wsb.data_ptr(), nb.value, sp)
        e2.record()
        _sync()
        t_comm.append(e0.elapsed_time(e1))
        t_all.append(e0.elapsed_time(e2))
    launches, tn, tms, tb = _abi.profile_read()
    _abi.profile_reset(False)
    ms = sum(t_all) / steps
    pairs = a.n * b.n
    return {"metric": "Pauli products collated/s", "value": ws * pairs / (ms / 1e3),
            "unit": "pairs/s", "n_gpus": ws, "steps": steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 keys / f64 coefficients",
            "data": "synthetic, seeded",
            "config": {"workload": "commutator: PauliSum<256,double> 16384 x 16384 windowed "
                                   "terms, canonicalize + cutoff(1e-14)",
                       "pairs": pairs, "emitted": emitted, "terms_out": n_out.value,
                       "commutator_ms": sum(t_comm) / steps,
                       "radix_passes_per_step": tn // steps,
                       "radix_pass_ms": tms / max(tn, 1),
                       "radix_pass_gbs": (tb / max(tn, 1)) / (tms / max(tn, 1) / 1e3) / 1e9},
            "gpu_launches": int(launches // steps)}
