"""The whole sharded collate on CPU ranks: two gloo ranks (127.0.0.1) run
ShardedPauliSum's own exchange_and_combine, global_terms, norm2 and
trim_global (MpiPauliSum.h:86-210) over a state whose device operations are
stood in for by the oracle (the packing restated in shard_ref), and the
result is checked against the oracle's canonical sum of the union: each
rank holds exactly the union's terms it owns, bit for bit."""
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


class OracleState:
    """The state interface ShardedPauliSum uses, on host planes with the
    oracle doing the arithmetic (test infrastructure)."""

    def __init__(self, p, oracle):
        self.p, self.o = p, oracle
        self.array_size = p.array_size

    def size(self):
        return self.p.n

    def shard_pack(self, ranks):
        import torch
        import shard_ref
        rec, counts = shard_ref.pack(self.p.x, self.p.z, self.p.flags, self.p.val, ranks)
        return torch.from_numpy(np.ascontiguousarray(rec).view(np.int64)), [int(c) for c in counts]

    def shard_unpack(self, recs):
        from paulib_b200.planes import Planes
        r = recs.numpy().view(np.uint64)
        aw = self.array_size
        self.p = Planes(np.ascontiguousarray(r[:, :aw].T), np.ascontiguousarray(r[:, aw:2 * aw].T),
                        r[:, 2 * aw].astype(np.uint8), r[:, 2 * aw + 1].copy().view(np.float64))

    def canonicalize(self):
        self.p = self.o.canonicalize(self.p)

    def frobenius_norm2(self):
        return self.o.frobenius_norm2(self.p)

    def max_abs(self):
        return float(np.abs(self.p.val).max()) if self.p.n else 0.0

    def count_above(self, t):
        return int((np.abs(self.p.val) >= t).sum())

    def cutoff(self, eps):
        self.p = self.o.cutoff(self.p, eps)


def _rank_main(rank, ws, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist

    import shard_ref
    from helpers import random_sum
    from oracle.oracle import Oracle
    from paulib_b200.planes import Planes
    from paulib_b200.sharded import ShardedPauliSum
    dist.init_process_group("gloo")
    try:
        o = Oracle()
        # 11 qubits and 3000 terms per rank: strings repeat within and across
        # the ranks' parts, so the exchange really merges
        parts = [random_sum(3000, 1, 40 + r, 11, "normal") for r in range(ws)]
        st = OracleState(parts[rank], o)
        sh = ShardedPauliSum(st, num_qubits=11)
        sh.exchange_and_combine()
        union = Planes(np.concatenate([p.x for p in parts], axis=1),
                       np.concatenate([p.z for p in parts], axis=1),
                       np.concatenate([p.flags for p in parts]),
                       np.concatenate([p.val for p in parts]))
        whole = o.canonicalize(union)
        own = shard_ref.owners(whole.x, whole.z, ws) == rank
        mine = st.p
        ok_terms = (mine.n == int(own.sum()) and np.array_equal(mine.x, whole.x[:, own]) and
                    np.array_equal(mine.z, whole.z[:, own]) and
                    np.array_equal(mine.flags, whole.flags[own]))
        # the same members meet in a different order than in the union's
        # single sort: equal within 1e-12 of the summed magnitudes
        scale = o.sort_and_combine(Planes(union.x, union.z, union.flags & np.uint8(1),
                                          np.abs(union.val)))
        sown = shard_ref.owners(scale.x, scale.z, ws) == rank
        ok_vals = ok_terms and bool(np.all(np.abs(mine.val - whole.val[own]) <=
                                           1e-12 * scale.val[sown]))
        gt = sh.global_terms()
        n2 = sh.norm2()
        want_n2 = o.frobenius_norm2(whole)
        max_terms = whole.n // 3
        sh.trim_global(max_terms)
        kept_min = float(np.abs(st.p.val).min()) if st.p.n else np.inf
        q.put((rank, ok_terms, ok_vals, gt == whole.n, abs(n2 - want_n2) <= 1e-12 * want_n2,
               st.p.n, kept_min, whole.n, max_terms,
               np.sort(np.abs(whole.val))[::-1].tolist()))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_collate_and_trim():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    # read the results before joining: a child exits only once its queued
    # result has been taken off the pipe
    res = sorted((q.get(timeout=300) for _ in range(2)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
    assert [p.exitcode for p in procs] == [0, 0]
    for _, ok_terms, ok_vals, ok_count, ok_norm, *_ in res:
        assert ok_terms and ok_vals and ok_count and ok_norm
    # trim_global: the kept terms are the globally largest magnitudes, at
    # least max_terms of them, ties at the threshold kept
    kept = sum(r[5] for r in res)
    thr = min(r[6] for r in res)
    mags, max_terms = np.array(res[0][9]), res[0][8]
    assert kept >= max_terms
    assert kept == int((mags >= thr).sum())
    assert kept <= int((mags >= mags[max_terms - 1]).sum())
