"""The sharded collate's device half on one GPU: pl_state_shard_pack against
the test-side restatement of the layout; several ranks emulated as
consecutive shards of one sum (their buckets exchanged by slicing) against
the oracle's canonical sum split by owner; and the real torch.distributed
path with one NCCL rank (exchange, global_terms, norm2, trim_global)."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

import shard_ref
from helpers import assert_keys_equal, bit_identical, random_sum
from paulib_b200.planes import Planes
from paulib_b200 import _abi
from paulib_b200 import propagation as PR

pytestmark = pytest.mark.gpu


def state_of(p: Planes):
    st = PR.State(p.array_size, max(p.n, 1 << 16))
    st.upload(p.x, p.z, p.flags, p.val)
    return st


def gpu_pack(st, n, ranks, words):
    import torch
    W = 2 * words + 2
    rec = torch.empty((max(n, 1), W), dtype=torch.int64, device="cuda")
    counts = (C.c_int64 * ranks)()
    _abi.check(st._lib.pl_state_shard_pack(st._h, ranks, rec.data_ptr(), n, counts))
    return rec[:n].cpu().numpy().view(np.uint64), np.array(list(counts))


@pytest.mark.parametrize("words,ranks", [(1, 1), (1, 3), (2, 2), (2, 8), (4, 5)])
def test_pack_matches_layout(cuda, words, ranks):
    p = random_sum(7000, words, 5 * words + ranks, None, "normal")
    with state_of(p) as st:
        rec, counts = gpu_pack(st, p.n, ranks, words)
    want, wc = shard_ref.pack(p.x, p.z, p.flags, p.val, ranks)
    assert np.array_equal(counts, wc)
    assert np.array_equal(rec, want)


def test_emulated_ranks_match_oracle(cuda, oracle):
    import torch
    ranks, words = 4, 1
    g = random_sum(40000, words, 99, 12, "normal")     # many duplicates across shards
    cuts = np.linspace(0, g.n, ranks + 1).astype(int)
    shards = [Planes(g.x[:, a:b], g.z[:, a:b], g.flags[a:b], g.val[a:b])
              for a, b in zip(cuts[:-1], cuts[1:])]
    packed = []
    for sh in shards:
        with state_of(sh) as st:
            packed.append(gpu_pack(st, sh.n, ranks, words))
    whole = oracle.canonicalize(g)
    own = shard_ref.owners(whole.x, whole.z, ranks)
    for r in range(ranks):
        parts = []
        for rec, counts in packed:
            start = int(counts[:r].sum())
            parts.append(rec[start:start + int(counts[r])])
        recv = torch.from_numpy(np.ascontiguousarray(np.concatenate(parts)).view(np.int64)).cuda()
        with PR.State(words, 1 << 16) as st:
            _abi.check(st._lib.pl_state_shard_unpack(st._h, recv.data_ptr(), recv.shape[0]))
            st.canonicalize()
            got = Planes(*st.download())
        sel = own == r
        want = Planes(whole.x[:, sel], whole.z[:, sel], whole.flags[sel], whole.val[sel])
        assert_keys_equal(got, want)
        assert bit_identical(got, want)


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_one_nccl_rank(cuda, oracle):
    import torch.distributed as dist

    from paulib_b200.sharded import ShardedPauliSum
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_port()))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        p = random_sum(30000, 2, 7, 80, "normal")
        with state_of(p) as st:
            sh = ShardedPauliSum(st, 80)
            sh.exchange_and_combine()
            got = Planes(*st.download())
            o = oracle.canonicalize(p)
            assert_keys_equal(got, o)
            assert sh.global_terms() == o.n
            assert abs(sh.norm2() - float((o.val ** 2).sum())) <= 1e-12 * float((o.val ** 2).sum())
            keep = 1000
            sh.trim_global(keep)
            kept = st.size()
            thr = np.sort(np.abs(o.val))[::-1][keep - 1]
            assert keep <= kept <= int((np.abs(o.val) >= thr * (1 - 1e-12)).sum())
    finally:
        dist.destroy_process_group()
