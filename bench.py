#!/usr/bin/env python
"""Pauli-sum hot-path benchmark on B200.

Default workload (the headline metric, "Pauli products collated/s"):
  PauliSum<64,double> product + canonicalize -- two sums of 4096 terms over
  20 active qubits (weight U{1..4}, op U{I,X,Y,Z}, coefficients N(0,1),
  seeded), i.e. 16,777,216 products collated per step through the fused
  pl_multiply_collate C-ABI call.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload product_collate|propagation|commutator]

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
    from oracle.oracle import Planes  # plain numpy container, no oracle code runs
    from paulib_b200 import workloads as W
    a, b = W.product_operands(seed=seed)
    return Planes(a.x, a.z, a.flags, a.val), Planes(b.x, b.z, b.flags, b.val)


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
    for items in (8, 12, 16):
        _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_ITEMS, items), "pl_set_tuning")
        step()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(3):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        tune_trials.append({"radix_items": items, "ms_per_step": t0.elapsed_time(t1) / 3})
    best = min(tune_trials, key=lambda t: t["ms_per_step"])
    tune_ms = [t["ms_per_step"] for t in tune_trials]
    best_items = best["radix_items"]
    if ws > 1:  # every rank uses rank 0's choice
        import torch.distributed as dist
        t = torch.tensor([best_items], device="cuda")
        dist.broadcast(t, 0)
        best_items = int(t.item())
    _abi.check(L.pl_set_tuning(_abi.PL_TUNE_RADIX_ITEMS, best_items), "pl_set_tuning")
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
        "config": {"workload": "product_collate: PauliSum<64,double> 4096 x 4096 product + "
                               "canonicalize, 20 active qubits, weight U{1..4}",
                   "terms_lhs": n, "terms_rhs": m, "products_per_step": total,
                   "terms_out": n_out, "array_size": 1, "parallelism": f"replicas x{ws}",
                   "l2": "flushed between steps (256 MB write outside the step events); "
                         "step working set 0.6 GB > 126 MB L2",
                   "tuned": {"radix_items": best_items,
                             "trials_ms_per_step": dict(zip(("8", "12", "16"), tune_ms))}},
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
        line["cpu_baseline"] = cpu_baseline_product()
    return line


def cpu_baseline_product(reps=3):
    """The reference build (oracle/_ref, OpenMP, all host threads) on the
    full product + canonicalize, `reps` times."""
    from oracle.oracle import Reference
    R = Reference()
    a, b = product_workload(seed=1)
    R.multiply_canonicalize(a, b)  # warm
    t0 = time.perf_counter()
    for _ in range(reps):
        R.multiply_canonicalize(a, b)
    dt = time.perf_counter() - t0
    return {"value": reps * a.n * b.n / dt, "unit": UNIT, "cores": R.threads,
            "kind": "reference",
            "sample": f"{reps} x full 4096x4096 multiply + canonicalize "
                      f"({dt:.1f} s, {os.path.basename(R.path)})"}


def run_reference(args, rank, ws):
    """Reference arm: the reference's CPU implementation, all host threads."""
    if rank != 0:
        return None
    from oracle.oracle import Planes, Reference
    R = Reference()
    a, b = product_workload(seed=1)
    total_budget = 90.0  # seconds for warm-up + timed steps
    rows = 256
    sub = lambda r: Planes(b.x[:, :r], b.z[:, :r], b.flags[:r], b.val[:r])  # noqa: E731
    t0 = time.perf_counter()
    R.multiply_canonicalize(a, sub(rows))
    t1 = time.perf_counter() - t0
    per_step = total_budget / max(1, args.steps + args.warmup)
    rows = int(max(16, min(b.n, rows * per_step / max(t1, 1e-3))))
    for _ in range(args.warmup):
        R.multiply_canonicalize(a, sub(rows))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        R.multiply_canonicalize(a, sub(rows))
    dt = time.perf_counter() - t0
    value = args.steps * a.n * rows / dt
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 keys / f64 coefficients",
        "data": "synthetic, seeded (numpy PCG64)", "impl": "reference",
        "config": {"workload": "product_collate: PauliSum<64,double> 4096 x 4096 product + "
                               "canonicalize, 20 active qubits, weight U{1..4}",
                   "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": R.threads, "kind": "reference",
                         "sample": f"per step: 4096 x {rows} product + canonicalize "
                                   f"(a row subset of the 4096 x 4096 workload)"},
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
