"""bench.py's multi-rank plumbing on CPU: two gloo ranks (127.0.0.1)
rendezvous through dist_setup, time is the max over ranks, barriers pass,
and the reference arm runs on rank 0 only (the other ranks exit without
work)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    try:
        r, local, w = bench.dist_setup()
        assert (r, local, w) == (rank, rank, ws)
        assert dist.get_backend() == "gloo"
        t = bench.max_over_ranks(10.0 + rank, w)
        bench.barrier(w)

        class Args:
            steps, warmup = 1, 3
        ref = bench.run_reference(Args(), r, w) if r != 0 else "rank0"
        q.put((rank, t, ref))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    assert codes == [0, 0], codes
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got[0] == (0, 11.0, "rank0")      # max over ranks seen by every rank
    assert got[1] == (1, 11.0, None)         # reference arm: no work off rank 0
