"""Autotuner for the batch form of propagation.

The tunables are the executor's: lanes (concurrent device-resident jobs),
CUDA-graph replay of rotation runs, and the dispatch order.  Each candidate
runs a seeded calibration set of jobs drawn from the same distribution as
the workload (not the workload itself); the fastest wins.  Results are kept
per (device, workload signature) in a JSON cache beside this file unless
PAULIB_B200_TUNE=force asks for a fresh search.
"""
from __future__ import annotations

import json
import os
import time

from . import batch as B

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, ".autotune.json")

DEFAULT_CANDIDATES = [
    {"lanes": 1, "graphs": True, "order": "longest"},
    {"lanes": 2, "graphs": True, "order": "longest"},
    {"lanes": 4, "graphs": False, "order": "longest"},
    {"lanes": 4, "graphs": True, "order": "longest"},
    {"lanes": 6, "graphs": False, "order": "longest"},
    {"lanes": 8, "graphs": False, "order": "longest"},
]


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:
        return "unknown"


def _load() -> dict:
    try:
        with open(CACHE) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(d: dict):
    try:
        with open(CACHE, "w") as fh:
            json.dump(d, fh, indent=1, sort_keys=True)
    except OSError:
        pass


def tune_batch(calibration, signature: str, candidates=None, repeats: int = 1) -> dict:
    """Best executor options for jobs like ``calibration`` (a list of
    workloads.Instance).  Returns {"lanes", "graphs", "order", "trials"}."""
    key = f"{_device_name()}|{signature}"
    cache = _load()
    if os.environ.get("PAULIB_B200_TUNE") != "force" and key in cache:
        return cache[key]
    js = B.JobSet(calibration)
    trials = []
    # one untimed pass so allocation and first-touch costs do not bias the first candidate
    B.batch_propagate(js, lanes=2, graphs=False)
    for c in candidates or DEFAULT_CANDIDATES:
        best = float("inf")
        for _ in range(repeats):
            t = time.perf_counter()
            B.batch_propagate(js, lanes=c["lanes"], graphs=c["graphs"], order=c["order"])
            best = min(best, time.perf_counter() - t)
        trials.append(dict(c, seconds=best))
    win = min(trials, key=lambda t: t["seconds"])
    out = {"lanes": win["lanes"], "graphs": win["graphs"], "order": win["order"],
           "trials": trials}
    cache[key] = out
    _store(cache)
    return out
