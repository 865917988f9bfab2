"""The exchange of the sharded collate on CPU: two gloo ranks (127.0.0.1)
pack their terms by owner (test-side restatement of the layout), exchange
them with exchange_records, and each rank receives exactly the terms it owns
from both ranks, source rank by source rank, in term order."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch
    import torch.distributed as dist

    import shard_ref
    from helpers import random_sum
    from paulib_b200.sharded import exchange_records
    dist.init_process_group("gloo")
    try:
        parts = [random_sum(300, 2, 70 + r, 100, "normal") for r in range(ws)]
        p = parts[rank]
        rec, counts = shard_ref.pack(p.x, p.z, p.flags, p.val, ws)
        recv, rc = exchange_records(torch.from_numpy(rec.view(np.int64)), list(counts))
        got = recv.numpy().view(np.uint64)
        want = []
        for src in range(ws):
            sr, sc = shard_ref.pack(parts[src].x, parts[src].z, parts[src].flags,
                                    parts[src].val, ws)
            start = int(sc[:rank].sum())
            want.append(sr[start:start + int(sc[rank])])
        want = np.concatenate(want)
        q.put((rank, bool(np.array_equal(got, want)), rc))
    finally:
        dist.destroy_process_group()


def test_two_rank_exchange():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert [p.exitcode for p in procs] == [0, 0]
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert all(ok for _, ok, _ in res)
    assert sum(sum(rc) for _, _, rc in res) == 600
