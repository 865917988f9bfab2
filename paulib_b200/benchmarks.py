"""Secondary benchmark workloads for bench.py (--workload ...).

propagation  Heisenberg propagation of sum_i Z_i through a 64-qubit, 20-layer
             brickwork CNOT+RX+RZ circuit, cutoff 1e-4, max weight 8, then
             zero_state_expectation (metric: propagations/s).
commutator   [A, B] of two PauliSum<256,double> of 16384 windowed terms,
             then canonicalize + cutoff(1e-14) (metric: pairs collated/s).
batch        independent propagations of mixed width (16/32/64/128 qubits)
             and depth (4..24 brickwork layers), single-Pauli observables,
             cutoff 1e-5, max weight 10: the batch executor with autotuned
             options against the plain one-instance-at-a-time path on the
             same jobs (metric: propagations/s).
serve        a Poisson stream of such jobs plus one heavy job (128 qubits,
             depth 40): the serving loop against plain FIFO service at the
             same arrivals (metric: propagations/s, with p50/p99 latency).
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
    if name == "batch":
        return _batch(args, rank, ws)
    if name == "serve":
        return _serve(args, rank, ws)
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
    # autotune: graph replay of the rotation chunks on or off (after one
    # untimed run each, which for graphs includes their capture)
    trial = {}
    for g in (False, True):
        st.use_graphs(g)
        once()
        _sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        once()
        e1.record()
        _sync()
        trial[g] = e0.elapsed_time(e1)
    graphs = min(trial, key=trial.get)
    st.use_graphs(graphs)
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
                       "rotations": int(r.n), "final_terms": final, "expectation": e,
                       "tuned": {"graphs": graphs,
                                 "trials_ms": {"off": trial[False], "on": trial[True]}}},
            "gpu_launches": int(launches // steps)}


def sub_circuit(circ: W.Circuit, layers: int) -> W.Circuit:
    """The first `layers` brickwork layers of a circuit (its ops and the
    rotations they use)."""
    n = circ.num_qubits
    per_layer = 2 * n  # rotations per layer (RX and RZ on every qubit)
    keep = [row for row in circ.ops
            if row[0] != W.OP_ROT or int(row[1]) < layers * per_layer]
    # CNOT rows of later layers come after the last kept rotation
    last = max(i for i, row in enumerate(keep) if row[0] == W.OP_ROT)
    ops = np.asarray(keep[: last + 1], np.int32).reshape(-1, 3)
    r = circ.rotations
    m = layers * per_layer
    rot = W.SoA(r.x[:, :m].copy(), r.z[:, :m].copy(), r.flags[:m].copy(), r.val[:m].copy(), n)
    return W.Circuit(rot, ops, n, {"layers": layers})


def propagation_bytes(log: np.ndarray, ops_reversed: np.ndarray, array_size: int,
                      n_obs: int) -> dict:
    """Byte models of one propagation from its gate log (terms in m,
    anticommuting k, terms out per rotation, processing order).

    design: the merge path's own traffic -- k_expand reads m terms and
    writes k children, the run merge reads and writes k, k_merge_reduce
    reads m + k and writes the out survivors: S*(2m + 4k + out) per
    rotation; a CNOT layer reads and writes the x, z and flags planes of
    its m terms.  survey: the reference algorithm's per-gate model,
    m*S + (m+k)*S + B_canon(m+k, out, b) with b = 2*64*AS + 1 key bits."""
    S = 16 * array_size + 9
    design = 0
    survey = 0
    b = 2 * 64 * array_size + 1
    kb = 8 * ((b + 63) // 64)
    passes = (b + 7) // 8
    size = n_obs
    prev_cnot = False
    for q, row in enumerate(ops_reversed):
        if row[0] == W.OP_ROT:
            m, k, out = (int(v) for v in log[q])
            if m == 0 and k == 0 and out == 0:
                continue
            design += S * (2 * m + 4 * k + out)
            survey += m * S + (m + k) * S + (m + k) * S + passes * (m + k) * 2 * (kb + 4) \
                + out * S
            size = out
            prev_cnot = False
        else:
            if not prev_cnot:
                design += 2 * (16 * array_size + 1) * size
            prev_cnot = True
    rows = log[log[:, 0] > 0]
    return {"design_bytes": int(design), "survey_bytes": int(survey),
            "rotations_logged": int(rows.shape[0]),
            "sum_m": int(rows[:, 0].sum()), "sum_k": int(rows[:, 1].sum()),
            "sum_out": int(rows[:, 2].sum()), "peak_terms": int(rows[:, 0].max(initial=0))}


def propagation_summary(seed=2, num_qubits=64, layers=20, steps=3, warmup=2, peak_gbs=None):
    """One propagation of sum_i Z_i through the brickwork circuit (cutoff 1e-4,
    max weight 8), CUDA-event timed per propagation (upload through
    zero_state_expectation), with graph replay autotuned, the gate log of an
    untimed run and the byte-model rooflines."""
    import torch
    obs, circ, tr = W.heisenberg_workload(seed=seed, num_qubits=num_qubits, layers=layers)
    r = circ.rotations
    st = PR.State(obs.array_size, 1 << 24)

    def once():
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        st.propagate(r.x, r.z, r.flags, r.val, circ.ops, tr["max_weight"], tr["cutoff"])
        return st.zero_state_expectation()

    def timed():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        e = once()
        e1.record()
        _sync()
        return e0.elapsed_time(e1), e

    trial = {}
    for g in (False, True):
        st.use_graphs(g)
        once()
        _sync()
        trial[g] = timed()[0]
    graphs = min(trial, key=trial.get)
    st.use_graphs(graphs)
    for _ in range(max(1, warmup)):
        once()
    _sync()
    times, e = [], None
    for _ in range(max(1, steps)):
        t, e = timed()
        times.append(t)
    final = st.size()
    # sizes per gate from an untimed run with the log on
    st.log_gates(True)
    once()
    log = st.gate_log()
    st.log_gates(False)
    st.close()
    ms = float(np.median(times))
    bm = propagation_bytes(log, circ.ops[::-1], obs.array_size, obs.n)
    out = {"workload": f"sum_i Z_i, {num_qubits} qubits, {layers} brickwork layers CNOT+RX+RZ, "
                       f"cutoff {tr['cutoff']:g}, max_weight {tr['max_weight']}",
           "ms_per_propagation": ms, "value": 1e3 / ms, "unit": "propagations/s",
           "steps": len(times), "final_terms": final, "expectation": e,
           "graphs": graphs, "trials_ms": {"graphs_off": trial[False], "graphs_on": trial[True]},
           "gate_counts": {k: bm[k] for k in ("rotations_logged", "sum_m", "sum_k", "sum_out",
                                              "peak_terms")}}
    if peak_gbs:
        gbs = bm["design_bytes"] / (ms / 1e3) / 1e9
        out["roofline"] = {
            "bound": "hbm", "unit": "GB/s", "peak": peak_gbs,
            "bytes_model": "per rotation S*(2m + 4k + out) (expand, run merge, merge-reduce), "
                           "per CNOT layer 2*(16*AS+1)*m; S = 16*AS + 9; sums over the logged "
                           "(m, k, out); re-sorts after CNOT layers not counted",
            "bytes_per_propagation": bm["design_bytes"], "achieved": gbs,
            "frac": gbs / peak_gbs}
        sgbs = bm["survey_bytes"] / (ms / 1e3) / 1e9
        out["survey_byte_model"] = {
            "bytes_model": "per rotation m*S + (m+k)*S + B_canon(m+k, out, b=129): the "
                           "reference algorithm's append + full sort per gate",
            "bytes_per_propagation": bm["survey_bytes"], "equivalent_gbs": sgbs,
            "equivalent_frac": sgbs / peak_gbs}
    return out


def run_commutator_with_output(args):
    """The commutator workload on this process's GPU (rank 0 operands); also
    returns the emitted terms' x and z planes (host copies) of the last step."""
    line, out, emitted = _commutator(args, 0, 1, keep=True)
    x, z, _, _ = out.to_host(emitted)
    return line, (x, z)


def _commutator(args, rank, ws, keep=False):
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
    kernels = {k: {"launches": c // steps, "ms_per_step": t / steps}
               for k, (c, t, _) in _abi.profile_report().items()}
    _abi.profile_reset(False)
    ms = sum(t_all) / steps
    pairs = a.n * b.n
    line = {"metric": "Pauli products collated/s", "value": ws * pairs / (ms / 1e3),
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
                       "radix_pass_gbs": (tb / max(tn, 1)) / (tms / max(tn, 1) / 1e3) / 1e9
                       if tn else None,
                       "collate_kernels": kernels},
            "gpu_launches": int(launches // steps)}
    if keep:
        return line, out, emitted
    return line


def _batch_jobs(args, rank):
    """Every stride-th job of the 512-job set (seeded per rank)."""
    stride = max(1, int(getattr(args, "batch_stride", 16)))
    return W.batch_instances(seed=4 + 1000 * rank)[::stride]


def _batch(args, rank, ws):
    from . import autotune
    from . import batch as B
    jobs = _batch_jobs(args, rank)
    js = B.JobSet(jobs)
    # calibration jobs: same distribution, another seed
    calib = W.batch_instances(seed=99, count=96)[::8]
    tuned = autotune.tune_batch(calib, "batch:16-128q,4-24 layers,1e-5,w10")
    opts = dict(lanes=tuned["lanes"], graphs=tuned["graphs"], order=tuned["order"])
    B.batch_propagate(js, **opts)  # warm-up pass (buffers, graphs)
    steps = max(1, min(args.steps, 3))
    t_b, t_p = [], []
    for _ in range(steps):
        _sync()
        t = time.perf_counter()
        rb = B.batch_propagate(js, **opts)
        t_b.append(time.perf_counter() - t)
    for _ in range(steps):
        _sync()
        t = time.perf_counter()
        rp = B.plain(js)
        t_p.append(time.perf_counter() - t)
    same = bool(np.array_equal(rb.expectation, rp.expectation) and
                np.array_equal(rb.final_terms, rp.final_terms))
    sb, sp = min(t_b), min(t_p)
    n = len(jobs)
    # the plain path runs one job at a time, so its per-job times are the
    # jobs' own: no schedule can finish before the longest one does
    dur = rp.end_s - rp.start_s
    longest = float(dur.max()) if n else 0.0
    return {"metric": "propagations/s", "value": ws * n / sb, "unit": "propagations/s",
            "n_gpus": ws, "steps": steps, "warmup": 1, "ms_per_step": sb * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 keys / f64 coefficients", "data": "synthetic, seeded",
            "config": {"workload": "batch: independent propagations, 16/32/64/128 qubits, "
                                   "4-24 brickwork layers, single-Pauli observables, "
                                   "cutoff 1e-5, max_weight 10",
                       "jobs": n, "stride_of_512": int(getattr(args, "batch_stride", 16)),
                       "tuned": {k: tuned[k] for k in ("lanes", "graphs", "order")},
                       "tuning_trials": tuned["trials"],
                       "plain_value": ws * n / sp, "plain_ms_per_step": sp * 1e3,
                       "speedup_vs_plain": sp / sb, "results_identical_to_plain": same,
                       "longest_job_s": longest,
                       "speedup_bound_by_longest_job": float(dur.sum()) / longest if longest
                       else None,
                       "peak_device_gb": rb.peak_bytes / 1e9,
                       "timing": "host wall clock around the call (all jobs' device work "
                                 "completes inside it), best of steps"}}


def _serve(args, rank, ws):
    from . import batch as B
    n = max(8, int(getattr(args, "serve_jobs", 40)))
    jobs = W.batch_instances(seed=7 + 1000 * rank, count=n)
    heavy = W.heavy_instance(seed=7 + 13 * rank)
    pos = n // 10
    jobs = jobs[:pos] + [heavy] + jobs[pos:]
    js0 = B.JobSet(jobs)
    # service capacity of the plain path on these jobs sets the arrival rate:
    # the offered load is a stated multiple of what the plain path can serve
    B.plain(js0)  # warm-up
    _sync()
    t = time.perf_counter()
    rp0 = B.plain(js0)
    service = time.perf_counter() - t
    load = float(getattr(args, "serve_load", 1.2))
    rate = load * len(jobs) / service
    arr = B.poisson_arrivals(len(jobs), rate, seed=17 + rank)
    js = B.JobSet(jobs, arr)
    lanes = int(getattr(args, "serve_lanes", 6))
    rs = B.serve(js, arr, lanes=lanes, graphs=False)
    rf = B.serve(js, arr, lanes=1, graphs=False)
    same = bool(np.array_equal(rs.expectation, rp0.expectation) and
                np.array_equal(rf.expectation, rp0.expectation))
    ls, lf = B.latency_percentiles(rs, arr), B.latency_percentiles(rf, arr)
    span_s = float(rs.end_s.max() - arr[0])
    span_f = float(rf.end_s.max() - arr[0])
    return {"metric": "propagations/s", "value": ws * len(jobs) / span_s,
            "unit": "propagations/s", "n_gpus": ws, "steps": 1, "warmup": 1,
            "ms_per_step": span_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 keys / f64 coefficients",
            "data": "synthetic, seeded Poisson arrivals",
            "config": {"workload": "serve: Poisson stream of batch-distribution jobs + 1 heavy "
                                   "(128 qubits, depth 40)",
                       "jobs": len(jobs), "arrival_rate_per_s": rate,
                       "offered_load_vs_plain": load, "lanes": lanes,
                       "latency": ls, "plain_fifo_latency": lf,
                       "plain_fifo_value": ws * len(jobs) / span_f,
                       "plain_service_s": service, "results_identical": same,
                       "peak_device_gb": rs.peak_bytes / 1e9}}


def main(argv=None) -> int:
    """A single workload run for profiling:

        python -m paulib_b200.benchmarks propagation [--layers 20] [--graphs 0|1] [--runs 1]

    propagates sum_i Z_i through the 64-qubit brickwork circuit (cutoff
    1e-4, max weight 8) `runs` times and prints the time of the last run,
    the final term count and the expectation."""
    import argparse
    import json
    import torch
    ap = argparse.ArgumentParser(description=main.__doc__.split("\n\n")[0])
    ap.add_argument("workload", choices=["propagation"])
    ap.add_argument("--layers", type=int, default=20)
    ap.add_argument("--graphs", type=int, default=0)
    ap.add_argument("--runs", type=int, default=1)
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=64, layers=a.layers)
    r = circ.rotations
    with PR.State(1, 1 << 24) as st:
        st.use_graphs(bool(a.graphs))
        for _ in range(max(1, a.runs)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            st.upload(obs.x, obs.z, obs.flags, obs.val)
            st.propagate(r.x, r.z, r.flags, r.val, circ.ops, tr["max_weight"], tr["cutoff"])
            e = st.zero_state_expectation()
            e1.record()
            _sync()
        print(json.dumps({"workload": f"propagation 64 qubits x {a.layers} layers",
                          "ms": e0.elapsed_time(e1), "final_terms": st.size(),
                          "expectation": e}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
