#!/usr/bin/env python
"""Pauli-sum hot-path benchmark on B200.

Default workload (the headline metric, "Pauli products collated/s"):
  PauliSum<64,double> product + canonicalize -- two sums of 4096 terms over
  20 active qubits (weight U{1..4}, op U{I,X,Y,Z}, coefficients N(0,1),
  seeded), i.e. 16,777,216 products collated per step through the fused
  pl_multiply_collate C-ABI call.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload product_collate|propagation|commutator|batch|serve]

At N = 1 the product_collate line also carries: parity of the timed output
against the reference build, the reference's own CUDA kernels timed beside
ours (gpu_comparator), the 64-qubit propagation with its byte-model roofline
and a reference CPU baseline on a circuit prefix (propagation), and the
served stream against plain FIFO service (served); --no-extras skips them.

Under torchrun (N > 1) every rank runs an independent instance of the
workload (weak scaling, no data-path collective); times are the max over
ranks.  --impl reference times the reference's own CPU implementation
(compiled from its headers into oracle/_ref) on the host cores, rank 0 only.

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events
on the launching stream with an L2 flush (256 MB write) between steps
outside the events; barrier + synchronize on both sides of the timed loop.
One JSON line is printed by rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Pauli products collated/s"
UNIT = "products/s"
L2_FLUSH_BYTES = 256 << 20


# ---------------------------------------------------------------------------
# process group
# ---------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, local, ws


def max_over_ranks(x: float, ws: int) -> float:
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "50"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        time.sleep(0.1)
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# roofline helpers
# ---------------------------------------------------------------------------
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(name: str):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", name + ".json")
    try:
        with open(p) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return None


def b_canon(n_in, n_out, bits, s_in=25, s_out=25):
    """Canonicalize byte model: inputs read once, P(b) 8-bit passes over
    (key + u32 index) read and written, outputs written once."""
    k = 8 * ((bits + 63) // 64)
    p = (bits + 7) // 8
    return n_in * s_in + p * n_in * 2 * (k + 4) + n_out * s_out


# ---------------------------------------------------------------------------
# product + collate (our arm)
# ---------------------------------------------------------------------------
def product_workload(seed):
    from paulib_b200 import workloads as W
    from paulib_b200.planes import Planes
    a, b = W.product_operands(seed=seed)
    return Planes(a.x, a.z, a.flags, a.val), Planes(b.x, b.z, b.flags, b.val)


def product_config(ws, n=4096, m=4096):
    """The workload description both arms print (identical by construction)."""
    return {"workload": "product_collate: PauliSum<64,double> 4096 x 4096 product + "
                        "canonicalize, 20 active qubits, weight U{1..4}",
            "terms_lhs": n, "terms_rhs": m, "products_per_step": n * m, "array_size": 1,
            "parallelism": f"replicas x{ws}",
            "l2": "flushed between steps (256 MB write outside the step events); "
                  "step working set 0.6 GB > 126 MB L2"}


def host_cpu():
    """Model name and thread count of this host (lscpu, else /proc/cpuinfo)."""
    name = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                name = ln.split(":", 1)[1].strip()
                break
    except (OSError, subprocess.SubprocessError):
        pass
    if name is None:
        try:
            with open("/proc/cpuinfo") as fh:
                for ln in fh:
                    if ln.startswith("model name"):
                        name = ln.split(":", 1)[1].strip()
                        break
        except OSError:
            pass
    return {"model": name, "nproc": os.cpu_count()}


def run_product_collate(args, rank, local, ws):
    import torch
    from paulib_b200 import _abi

    torch.cuda.set_device(local)
    L = _abi.lib()
    a, b = product_workload(seed=1 + rank)
    n, m = a.n, b.n
    total = n * m
    da = _abi.DeviceSum.from_host(a.x, a.z, a.flags, a.val)
    db = _abi.DeviceSum.from_host(b.x, b.z, b.flags, b.val)
    out = _abi.DeviceSum(1, total)
    nb = C.c_size_t()
    _abi.check(L.pl_multiply_collate_workspace_size(1, n, m, C.byref(nb)))
    ws_buf = _abi.workspace(nb.value)
    opts = _abi.CollateOpts(_abi.PL_COLLATE_CANONICALIZE, 0, 0.0, _abi.UINT64_MAX)
    stream = torch.cuda.current_stream()
    sp = int(stream.cuda_stream)
    cnt = C.c_int64()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def step(src_a=da, src_b=db, dst=out):
        _abi.check(L.pl_multiply_collate(1, *src_a.ptrs(), n, *src_b.ptrs(), m, *dst.ptrs(),
                                         dst.capacity, C.byref(cnt), C.byref(opts),
                                         ws_buf.data_ptr(), nb.value, sp), "pl_multiply_collate")
        return cnt.value

    for _ in range(args.warmup):
        n_out = step()
    torch.cuda.synchronize()

    # ---- autotune: keys per thread of the digit pass -------------------
    tune_trials = []
    # (L2 prefetch one wave ahead / off) x keys per thread at a look-back
    # window of 4, then the window at the best of those; --tune fixes one
    # combination (profiling runs: fewer trial collates)
    def trial(items, prefetch, window, wide=-1, backoff=64, gather=-1):
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_FOLD_GATHER, gather), "pl_set_tuning")
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_BACKOFF, backoff), "pl_set_tuning")
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_ITEMS, items), "pl_set_tuning")
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_PREFETCH, prefetch), "pl_set_tuning")
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_WINDOW, window), "pl_set_tuning")
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_WIDE, wide), "pl_set_tuning")
        step()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(3):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        tune_trials.append({"radix_items": items, "radix_prefetch": prefetch,
                            "radix_window": window, "radix_wide": wide,
                            "radix_backoff": backoff, "fold_gather": gather,
                            "ms_per_step": t0.elapsed_time(t1) / 3})

    if args.tune:
        trial(*(int(v) for v in args.tune.split(",")))
    else:
        for wide in (-1, 1):  # 8-bit / 10-bit digits (10-bit needs >= 12 keys per thread)
            for prefetch in (0, -1):
                for items in ((8, 12, 16) if wide < 0 else (12, 16)):
                    trial(items, prefetch, 4, wide)
        b0 = min(tune_trials, key=lambda t: t["ms_per_step"])
        for window in (2, 8, 16):
            trial(b0["radix_items"], b0["radix_prefetch"], window, b0["radix_wide"])
        b1 = min(tune_trials, key=lambda t: t["ms_per_step"])
        for backoff in (1, 4, 16):
            trial(b1["radix_items"], b1["radix_prefetch"], b1["radix_window"], b1["radix_wide"],
                  backoff)
        b2 = min(tune_trials, key=lambda t: t["ms_per_step"])
        trial(b2["radix_items"], b2["radix_prefetch"], b2["radix_window"], b2["radix_wide"],
              b2["radix_backoff"], 1)
    best = min(tune_trials, key=lambda t: t["ms_per_step"])
    best_items, best_pf, best_w, best_wide, best_bo, best_g = (
        best["radix_items"], best["radix_prefetch"], best["radix_window"], best["radix_wide"],
        best["radix_backoff"], best["fold_gather"])
    if ws > 1:  # every rank uses rank 0's choice
        import torch.distributed as dist
        t = torch.tensor([best_items, best_pf, best_w, best_wide, best_bo, best_g], device="cuda")
        dist.broadcast(t, 0)
        best_items, best_pf, best_w, best_wide, best_bo, best_g = (int(v) for v in t.tolist())
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_ITEMS, best_items), "pl_set_tuning")
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_PREFETCH, best_pf), "pl_set_tuning")
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_WINDOW, best_w), "pl_set_tuning")
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_WIDE, best_wide), "pl_set_tuning")
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_BACKOFF, best_bo), "pl_set_tuning")
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_FOLD_GATHER, best_g), "pl_set_tuning")
    for _ in range(args.warmup):
        n_out = step()
    torch.cuda.synchronize()

    # ---- device-resident timing ---------------------------------------
    _abi.profile_reset(timing=True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for e0, e1 in evs:
            flush.zero_()
            e0.record(stream)
            n_out = step()
            e1.record(stream)
        torch.cuda.synchronize()
    barrier(ws)
    launches, timed_n, timed_ms, timed_bytes = _abi.profile_read()
    kernels = {k: {"launches": c, "ms_per_step": t / args.steps}
               for k, (c, t, _) in _abi.profile_report().items()}
    _abi.profile_reset(timing=False)
    step_ms = [e0.elapsed_time(e1) for e0, e1 in evs]
    t_ms = max_over_ranks(sum(step_ms), ws)
    ms_per_step = t_ms / args.steps
    value = ws * total * args.steps / (t_ms / 1e3)

    # ---- end to end through the C ABI with host buffers ----------------
    # Every step copies its operands in from pinned host memory, runs
    # pl_multiply_collate (synchronous, like the reference's call) and reads
    # its collated sum back into pinned host memory.  The read-back of step k
    # runs on a copy stream into its own host buffer while step k + 1
    # computes into the other device buffer (results double-buffered); the
    # timed region ends after the last read-back.
    ref_vals = out.val[:n_out].cpu()
    pin = lambda t: t.pin_memory()  # noqa: E731
    ha = [pin(t.cpu()) for t in (da.x, da.z, da.flags, da.val)]
    hb = [pin(t.cpu()) for t in (db.x, db.z, db.flags, db.val)]
    ea = _abi.DeviceSum(1, n)
    eb = _abi.DeviceSum(1, m)
    dev_out = [out, _abi.DeviceSum(1, total)]
    host_out = [[torch.empty(total, dtype=torch.int64, pin_memory=True),
                 torch.empty(total, dtype=torch.int64, pin_memory=True),
                 torch.empty(total, dtype=torch.uint8, pin_memory=True),
                 torch.empty(total, dtype=torch.float64, pin_memory=True)] for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    h2d = sum(t.numel() * t.element_size() for t in ha + hb)
    d2h = []

    def h2d_inputs():
        for dst, src in zip((ea.x, ea.z, ea.flags, ea.val), ha):
            dst.view(-1)[: src.numel()].copy_(src.view(-1), non_blocking=True)
        for dst, src in zip((eb.x, eb.z, eb.flags, eb.val), hb):
            dst.view(-1)[: src.numel()].copy_(src.view(-1), non_blocking=True)

    def e2e_step(i, first, more):
        # step i's operands were copied in before it (by step i - 1 when it
        # has one): issued ahead of step i - 1's result read-back, they do
        # not queue behind it on a copy engine
        b = i % 2
        stream.wait_event(copied[b])  # the read-back of step i - 2 left dev_out[b]
        if first:
            h2d_inputs()
        k = step(ea, eb, dev_out[b])
        if more:
            h2d_inputs()  # the next step's operands
        o = dev_out[b]
        outs = (o.x.view(-1)[:k], o.z.view(-1)[:k], o.flags[:k], o.val[:k])
        copy_stream.wait_stream(stream)
        nbytes = 0
        with torch.cuda.stream(copy_stream):
            for dst, src in zip(host_out[b], outs):
                dst[:k].copy_(src, non_blocking=True)
                nbytes += src.numel() * src.element_size()
            copied[b].record(copy_stream)
        return nbytes

    nw = max(2, args.warmup // 2)
    for i in range(nw):
        e2e_step(i, i == 0, i + 1 < nw)
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(3, args.steps // 4)
    e0.record(stream)
    for i in range(e2e_steps):
        d2h.append(e2e_step(i, i == 0, i + 1 < e2e_steps))
    stream.wait_stream(copy_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), ws)
    e2e_value = ws * total * e2e_steps / (e2e_ms / 1e3)
    # the last step's result as read back equals the device-resident run's
    assert d2h[-1] == n_out * 25, "e2e read-back size"
    assert torch.equal(host_out[(e2e_steps - 1) % 2][3][:n_out], ref_vals), \
        "e2e result differs from the device-timed run"

    # ---- roofline of the dominant kernel (onesweep digit pass) ---------
    peak, peak_kind = measured_peaks()
    per_launch_ms = timed_ms / max(timed_n, 1)
    per_launch_bytes = timed_bytes / max(timed_n, 1)
    achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
    # DRAM bytes per launch from the committed ncu capture of this workload,
    # scaled by this run's algorithmic bytes per launch over the captured one
    prof = profile_traffic("radix_pass_product_collate")
    traffic = None
    if prof and prof.get("dram_bytes_per_launch") and prof.get("algorithmic_bytes_per_launch"):
        traffic = prof["dram_bytes_per_launch"] * (per_launch_bytes /
                                                   prof["algorithmic_bytes_per_launch"])
    bits = 41
    pipe_bytes = b_canon(total, n_out, bits)
    pipe_gbs = pipe_bytes / (ms_per_step / 1e3) / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 keys / f64 coefficients",
        "data": "synthetic, seeded (numpy PCG64); shapes and distributions of the "
                "product+collate benchmark",
        "config": product_config(ws, n, m),
        "result": {"terms_out": n_out},
        "tuned": {"radix_items": best_items, "radix_l2_prefetch": best_pf == 0,
                  "radix_lookback_window": best_w, "radix_digit_bits": 10 if best_wide > 0 else 8,
                  "radix_lookback_hot_polls": best_bo, "fold_gathers_coefficients": best_g > 0,
                  "trials_ms_per_step": {
                      ("prefetch" if t["radix_prefetch"] == 0 else "plain")
                      + f"-{t['radix_items']}-w{t['radix_window']}"
                      + ("-d10" if t["radix_wide"] > 0 else "-d8")
                      + f"-b{t['radix_backoff']}"
                      + ("-fg" if t["fold_gather"] > 0 else ""): t["ms_per_step"]
                      for t in tune_trials}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": int(statistics.mean(d2h)),
                "path": "pinned host planes -> H2D -> pl_multiply_collate (C ABI) -> D2H of "
                        "the collated sum; each read-back overlaps the next step's compute "
                        "(double-buffered results)"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "k_radix_pass (onesweep digit pass)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "launches_timed": timed_n, "ms_per_launch": per_launch_ms},
        "pipeline_roofline": {"bytes_model": "B_canon(n_in, n_out, b=41)",
                              "bytes_per_step": pipe_bytes, "achieved": pipe_gbs,
                              "peak": peak, "frac": pipe_gbs / peak, "unit": "GB/s"},
        "kernels": kernels,
        "clocks": clk.summary(),
    }
    if ws == 1 and rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"], ref = cpu_baseline_product()
        line["parity"] = product_parity(out, n_out, ref)
    if ws == 1 and not args.no_extras:
        line["gpu_comparator"] = gpu_comparator(da, db, n, m, stream)
        del out, dev_out, ea, eb, host_out
        torch.cuda.empty_cache()
        line["propagation"] = propagation_extra(args, peak)
        line["served"] = served_extra(args)
        line["batch"] = batch_extra(args)
        line["commutator"] = commutator_extra(args, peak)
    return line


def cpu_baseline_product(reps=3):
    """The reference build (oracle/_ref, OpenMP, all host threads) on the
    full product + canonicalize, `reps` times; also returns its result (the
    parity check of the timed output)."""
    from oracle.oracle import Reference
    R = Reference()
    a, b = product_workload(seed=1)
    R.multiply_canonicalize(a, b)  # warm
    t0 = time.perf_counter()
    for _ in range(reps):
        ref = R.multiply_canonicalize(a, b)
    dt = time.perf_counter() - t0
    return ({"value": reps * a.n * b.n / dt, "unit": UNIT, "cores": R.threads,
             "kind": "reference", "cpu": host_cpu(),
             "sample": f"{reps} x full 4096x4096 multiply + canonicalize "
                       f"({dt:.1f} s, {os.path.basename(R.path)})"}, ref)


def product_parity(out, n_out, ref):
    """The device-timed step's output against the reference build's result
    on the same operands: strings, phases and order exact; coefficients
    within 1e-12 relative of max(|c|, 1) (the reference's -ffast-math build
    reassociates its segment sums)."""
    import numpy as np
    got = out.to_host(n_out)
    keys = (n_out == ref.n and np.array_equal(got[0], ref.x) and np.array_equal(got[1], ref.z)
            and np.array_equal(got[2], ref.flags))
    rel = float((np.abs(got[3] - ref.val) / np.maximum(np.abs(ref.val), 1.0)).max()) \
        if keys and n_out else None
    ok = bool(keys and rel is not None and rel <= 1e-12)
    return {"vs": "reference build (oracle/_ref) on the rank-0 operands", "ok": ok,
            "terms": int(n_out), "reference_terms": int(ref.n), "strings_exact": bool(keys),
            "max_rel_err": rel, "tolerance": "1e-12 of max(|c|, 1)"}


def gpu_comparator(da, db, n, m, stream, reps=10):
    """The reference's own CUDA kernels (baseline/_ref/libpaulib_refgpu.so:
    src/gpu/gpu_mul.cu and gpu_commutator.cu built unchanged for sm_100a by
    baseline/Makefile) against this library's drop-ins with the same C
    signatures, on the same device operands, CUDA-event timed (median of
    `reps` launches after 3 untimed)."""
    import torch
    from paulib_b200 import _abi
    from paulib_b200 import workloads as W
    path = os.path.join(ROOT, "baseline", "_ref", "libpaulib_refgpu.so")
    if not os.path.exists(path):
        return {"unavailable": "baseline/_ref/libpaulib_refgpu.so not built (make -C baseline)"}
    R = C.CDLL(path)  # RTLD_LOCAL: its launch_gpu_* stay apart from ours
    L = _abi.lib()
    sp = int(stream.cuda_stream)
    VP = C.c_void_p
    for lib in (R, L):
        lib.launch_gpu_mul_soa.restype = None
        lib.launch_gpu_mul_soa.argtypes = [C.c_int] + [VP] * 12 + [C.c_int, C.c_int, VP]
        lib.launch_gpu_commutator_soa.restype = None
        lib.launch_gpu_commutator_soa.argtypes = ([C.c_int, C.c_int] + [VP] * 13 +
                                                  [C.c_int, C.c_int, C.c_longlong, VP])

    def timeit(fn, pre=None):
        for _ in range(3):
            if pre:
                pre()
            fn()
        ts = []
        for _ in range(reps):
            if pre:
                pre()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    res = {"reference_build": "src/gpu/gpu_mul.cu + gpu_commutator.cu, nvcc "
                              "-gencode arch=compute_100a,code=sm_100a --use_fast_math -O3"}
    # outer product, 4096 x 4096 at AS = 1 (the reference's launcher needs
    # only n*m output slots; its kernel writes one term per pair)
    prod = _abi.DeviceSum(1, n * m)
    same = True
    outs = {}
    for name, lib in (("reference", R), ("ours", L)):
        t = timeit(lambda lib=lib: lib.launch_gpu_mul_soa(1, *da.ptrs(), *db.ptrs(),
                                                          *prod.ptrs(), n, m, sp))
        outs[name] = t
        h = prod.val[: n * m].clone()
        if name == "reference":
            ref_val = h
        else:
            same = bool(torch.equal(ref_val, h))
    res["multiply"] = {"shape": f"{n} x {m}, array_size 1", "reference_ms": outs["reference"],
                       "ours_ms": outs["ours"], "speedup": outs["reference"] / outs["ours"],
                       "products_per_s_ours": n * m / (outs["ours"] / 1e3),
                       "write_gbs_ours": n * m * 25 / (outs["ours"] / 1e3) / 1e9,
                       "values_identical": same}
    del prod, ref_val, h
    # commutator, 16384 x 16384 at 256 qubits (AS = 4): the reference's
    # kernel claims output slots with an unchecked atomic counter, so its
    # output planes get the only capacity that is safe by construction, n*m
    a, b = W.window_sums(seed=3)
    ca = _abi.DeviceSum.from_host(a.x, a.z, a.flags, a.val)
    cb = _abi.DeviceSum.from_host(b.x, b.z, b.flags, b.val)
    cap = a.n * b.n
    try:
        big = _abi.DeviceSum(4, cap)
    except RuntimeError as e:  # allocation
        res["commutator"] = {"unavailable": f"n*m output planes: {e}"}
        return res
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    counts = {}
    for name, lib in (("reference", R), ("ours", L)):
        t = timeit(lambda lib=lib: lib.launch_gpu_commutator_soa(
            4, 0, *ca.ptrs(), *cb.ptrs(), *big.ptrs(), cnt.data_ptr(), a.n, b.n, cap, sp),
            pre=cnt.zero_)
        outs[name] = t
        counts[name] = int(cnt.item())
    res["commutator"] = {"shape": f"{a.n} x {b.n}, array_size 4 (256 qubits, windowed)",
                         "reference_ms": outs["reference"], "ours_ms": outs["ours"],
                         "speedup": outs["reference"] / outs["ours"],
                         "pairs_per_s_ours": a.n * b.n / (outs["ours"] / 1e3),
                         "emitted": counts["ours"],
                         "emitted_equal": counts["ours"] == counts["reference"],
                         "note": "ours includes its stream-ordered look-back scratch "
                                 "(allocate, clear, free) and emits in deterministic order"}
    del big
    torch.cuda.empty_cache()
    return res


def propagation_extra(args, peak):
    """Propagation (sum_i Z_i, 64 qubits, 20 layers): GPU timing with the
    gate-log rooflines, plus the reference build timed on a prefix of the
    circuit beside the GPU on the same prefix."""
    from paulib_b200 import benchmarks
    from paulib_b200 import propagation as PR
    from paulib_b200 import workloads as W
    out = benchmarks.propagation_summary(steps=3, warmup=2, peak_gbs=peak)
    if args.no_cpu_baseline:
        return out
    from oracle.oracle import Reference
    from paulib_b200.planes import Planes
    layers = int(args.prop_cpu_layers)
    obs, circ, tr = W.heisenberg_workload(seed=2, num_qubits=64, layers=20)
    sub = benchmarks.sub_circuit(circ, layers)
    R = Reference()
    r = sub.rotations
    t0 = time.perf_counter()
    ref = R.propagate(Planes(obs.x, obs.z, obs.flags, obs.val), Planes(r.x, r.z, r.flags, r.val),
                      sub.ops, max_weight=tr["max_weight"], cutoff=tr["cutoff"])
    cpu_s = time.perf_counter() - t0
    import torch
    with PR.State(1, 1 << 20) as st:
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        st.propagate(r.x, r.z, r.flags, r.val, sub.ops, tr["max_weight"], tr["cutoff"])
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        st.upload(obs.x, obs.z, obs.flags, obs.val)
        st.propagate(r.x, r.z, r.flags, r.val, sub.ops, tr["max_weight"], tr["cutoff"])
        e1.record()
        torch.cuda.synchronize()
        gpu_ms = e0.elapsed_time(e1)
        same = st.size() == ref.n
    out["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "propagations/s of the prefix",
                           "cores": R.threads, "kind": "reference", "cpu": host_cpu(),
                           "sample": f"the first {layers} of the 20 layers "
                                     f"({r.n} rotations): {cpu_s:.2f} s; the GPU on the same "
                                     f"prefix {gpu_ms:.2f} ms",
                           "gpu_ms_same_prefix": gpu_ms,
                           "speedup_same_prefix": cpu_s * 1e3 / gpu_ms,
                           "terms_equal": bool(same)}
    return out


def served_extra(args):
    """Served stream (Poisson arrivals of mixed-batch jobs + one heavy job)
    against plain FIFO service at the same arrivals."""
    from paulib_b200 import benchmarks
    ns = argparse.Namespace(serve_jobs=args.serve_jobs, serve_lanes=args.serve_lanes,
                            serve_load=args.serve_load)
    line = benchmarks.run("serve", ns, 0, torch_local_rank(), 1)
    c = line["config"]
    return {"workload": c["workload"], "jobs": c["jobs"], "value": line["value"],
            "unit": line["unit"], "arrival_rate_per_s": c["arrival_rate_per_s"],
            "offered_load_vs_plain": c["offered_load_vs_plain"], "lanes": c["lanes"],
            "latency": c["latency"], "plain_fifo": {"value": c["plain_fifo_value"],
                                                    "latency": c["plain_fifo_latency"]},
            "speedup_vs_plain_fifo": line["value"] / c["plain_fifo_value"],
            "results_identical": c["results_identical"],
            "peak_device_gb": c["peak_device_gb"]}


def batch_extra(args):
    """Batched propagation (every 16th job of the 512-job mixed set, the
    autotuned executor) against the plain one-at-a-time path on the same
    jobs, with the bound the longest job puts on any schedule."""
    from paulib_b200 import benchmarks
    ns = argparse.Namespace(batch_stride=args.batch_stride, steps=1, warmup=1)
    line = benchmarks.run("batch", ns, 0, torch_local_rank(), 1)
    c = line["config"]
    return {"workload": c["workload"], "jobs": c["jobs"], "stride_of_512": c["stride_of_512"],
            "value": line["value"], "unit": line["unit"], "plain_value": c["plain_value"],
            "speedup_vs_plain": c["speedup_vs_plain"],
            "longest_job_s": c["longest_job_s"],
            "speedup_bound_by_longest_job": c["speedup_bound_by_longest_job"],
            "results_identical_to_plain": c["results_identical_to_plain"],
            "tuned": c["tuned"], "timing": c["timing"]}


def commutator_extra(args, peak):
    """Commutator + canonicalize + cutoff(1e-14) of two 16384-term sums on
    256 qubits (windowed supports, array_size 4), with the collate's byte
    models: B_canon over the plain key's varying bits (the reference
    algorithm's sort), and the digit passes actually run."""
    import numpy as np
    from paulib_b200 import benchmarks
    ns = argparse.Namespace(steps=10, warmup=3)
    line, emitted_planes = benchmarks.run_commutator_with_output(ns)
    c = line["config"]
    x, z = emitted_planes
    var = 0
    for w in range(x.shape[0]):
        var += bin(int(np.bitwise_or.reduce(x[w]) ^ np.bitwise_and.reduce(x[w]))).count("1")
        var += bin(int(np.bitwise_or.reduce(z[w]) ^ np.bitwise_and.reduce(z[w]))).count("1")
    bits = var + 1  # the phase after the sign fold
    s_term = 16 * 4 + 9
    collate_ms = line["ms_per_step"] - c["commutator_ms"]
    bc = b_canon(c["emitted"], c["terms_out"], bits, s_term, s_term)
    return {"workload": c["workload"], "pairs": c["pairs"], "emitted": c["emitted"],
            "terms_out": c["terms_out"], "ms_per_step": line["ms_per_step"],
            "commutator_ms": c["commutator_ms"], "collate_ms": collate_ms,
            "value": line["value"], "unit": line["unit"],
            "digit_passes_per_step": c["radix_passes_per_step"],
            "collate_kernels": c["collate_kernels"],
            "digit_pass_ms": c["radix_pass_ms"], "digit_pass_gbs": c["radix_pass_gbs"],
            "plain_key_varying_bits": bits,
            "b_canon": {"bytes_model": "B_canon(emitted, terms_out, b) with S = 73 B",
                        "bits": bits, "bytes": bc,
                        "equivalent_gbs": bc / (collate_ms / 1e3) / 1e9,
                        "equivalent_frac": bc / (collate_ms / 1e3) / 1e9 / peak}}


def torch_local_rank():
    return int(os.environ.get("LOCAL_RANK", "0"))


def run_reference(args, rank, ws):
    """Reference arm: the reference's CPU implementation (oracle/_ref, its
    own header-only code with its flags), all host threads, on the same
    workload and config as our arm.  Each step is the full 4096 x 4096
    product + canonicalize unless the whole run would exceed a few minutes;
    then each step takes the same row subset of the rhs (stated in
    cpu_baseline.sample), and products/s is counted over the rows done."""
    if rank != 0:
        return None
    from oracle.oracle import Reference
    from paulib_b200.planes import Planes
    R = Reference()
    a, b = product_workload(seed=1)
    budget_s = 240.0
    t0 = time.perf_counter()
    R.multiply_canonicalize(a, b)  # first warm-up step doubles as the size probe
    t_full = time.perf_counter() - t0
    rows = b.n
    if t_full * (args.steps + args.warmup) > budget_s:
        rows = int(max(64, b.n * budget_s / (t_full * (args.steps + args.warmup))))
    sub = Planes(b.x[:, :rows], b.z[:, :rows], b.flags[:rows], b.val[:rows])
    for _ in range(args.warmup - 1):
        R.multiply_canonicalize(a, sub)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        R.multiply_canonicalize(a, sub)
    dt = time.perf_counter() - t0
    value = args.steps * a.n * rows / dt
    sample = ("per step: the full 4096 x 4096 product + canonicalize" if rows == b.n else
              f"per step: 4096 x {rows} product + canonicalize (the first {rows} rhs rows; "
              f"the full step takes {t_full:.2f} s here)")
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 keys / f64 coefficients",
        "data": "synthetic, seeded (numpy PCG64); shapes and distributions of the "
                "product+collate benchmark",
        "impl": "reference", "config": product_config(ws),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": R.threads, "kind": "reference",
                         "cpu": host_cpu(), "sample": sample,
                         "build": os.path.basename(R.path)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="product_collate",
                    choices=["product_collate", "propagation", "commutator", "batch", "serve"])
    ap.add_argument("--batch-stride", type=int, default=16,
                    help="batch workload: every n-th job of the 512-job set")
    ap.add_argument("--serve-jobs", type=int, default=40)
    ap.add_argument("--serve-lanes", type=int, default=6)
    ap.add_argument("--serve-load", type=float, default=1.2,
                    help="serve workload: arrival rate as a multiple of the plain path's capacity")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune", default="",
                    help="ITEMS,PREFETCH,WINDOW[,WIDE[,BACKOFF[,FOLD_GATHER]]]: fix the "
                         "digit-pass tuning instead of timing the combinations "
                         "(e.g. 16,0,4 or 12,0,8,-1,16,1)")
    ap.add_argument("--no-extras", action="store_true",
                    help="product_collate: skip the GPU comparator, propagation and served "
                         "sub-objects")
    ap.add_argument("--prop-cpu-layers", type=int, default=6,
                    help="propagation sub-object: layers of the circuit prefix the reference "
                         "build is timed on")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank, local, ws = dist_setup()
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, ws)
        elif args.workload == "product_collate":
            line = run_product_collate(args, rank, local, ws)
        else:
            from paulib_b200 import benchmarks
            line = benchmarks.run(args.workload, args, rank, local, ws)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
