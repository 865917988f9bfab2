"""Sharded Pauli sums across ranks: the hash-owned layout of the reference's
MPI add-on (MpiPauliSum.h), with one process per GPU and torch.distributed
(NCCL over NVLink / NVSwitch) for the exchange.

Every term is owned by rank FNV-1a(x, z) mod world_size (the phase is
excluded, so P, -P and iP meet on one rank).  exchange_and_combine packs the
local terms into per-owner buckets on the device (pl_state_shard_pack), moves
them with one all-to-all of term records, unpacks what arrived
(pl_state_shard_unpack) and canonicalizes locally: afterwards the ranks'
sums are disjoint and each is canonical, and together they are the global
canonical sum.  global_terms, norm2 and trim_global follow the reference's
collective definitions (MpiPauliSum.h:86-97, 187-210).
"""
from __future__ import annotations

from .propagation import State


def record_words(array_size: int) -> int:
    """u64 words of one term record: x[0..AS), z[0..AS), flags, value bits."""
    return 2 * int(array_size) + 2


def exchange_records(send, counts, group=None):
    """All-to-all of term records.  send: (n, W) int64 tensor whose rows are
    grouped by destination rank, counts[r] rows for rank r.  Returns the
    received (m, W) tensor (rows from rank 0 first, then rank 1, ...) and the
    per-source counts.  Works on CUDA tensors (NCCL) and CPU tensors (gloo)."""
    import torch
    import torch.distributed as dist
    ws = dist.get_world_size(group)
    assert len(counts) == ws
    dev = send.device
    sc = torch.tensor([int(c) for c in counts], dtype=torch.int64, device=dev)
    rc = torch.empty_like(sc)
    dist.all_to_all_single(rc, sc, group=group)
    recv_counts = [int(v) for v in rc.tolist()]
    recv = torch.empty((sum(recv_counts), send.shape[1]), dtype=send.dtype, device=dev)
    dist.all_to_all_single(recv, send[: sum(int(c) for c in counts)].contiguous(),
                           output_split_sizes=recv_counts,
                           input_split_sizes=[int(c) for c in counts], group=group)
    return recv, recv_counts


class ShardedPauliSum:
    """This rank's share of a sum distributed over the ranks of `group`.

    `state` is a propagation.State (device-resident); the class uses only its
    size, shard_pack, shard_unpack, canonicalize, frobenius_norm2, max_abs,
    count_above and cutoff."""

    def __init__(self, state: State, num_qubits: int, group=None):
        import torch.distributed as dist
        self.state = state
        self.num_qubits = int(num_qubits)
        self.group = group
        self.rank = dist.get_rank(group)
        self.ranks = dist.get_world_size(group)

    def _allreduce(self, value, op):
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([value], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op, group=self.group)
        return float(t.item())

    def exchange_and_combine(self):
        """Route every local term to its owner, then combine locally
        (MpiPauliSum.h:101-181)."""
        send, counts = self.state.shard_pack(self.ranks)
        recv, _ = exchange_records(send, counts, self.group)
        self.state.shard_unpack(recv)
        self.state.canonicalize()

    def global_terms(self) -> int:
        import torch.distributed as dist
        return int(self._allreduce(self.state.size(), dist.ReduceOp.SUM))

    def norm2(self) -> float:
        import torch.distributed as dist
        return self._allreduce(self.state.frobenius_norm2(), dist.ReduceOp.SUM)

    def trim_global(self, max_terms: int):
        """Keep (at least) the max_terms globally largest |c|: bisection on the
        magnitude threshold with global counts, then a local cutoff; ties at
        the threshold are kept (MpiPauliSum.h:187-210)."""
        import torch.distributed as dist
        if self.global_terms() <= max_terms:
            return
        st = self.state
        hi = self._allreduce(st.max_abs(), dist.ReduceOp.MAX)
        lo = 0.0

        def count_at(t):
            return int(self._allreduce(float(st.count_above(t)), dist.ReduceOp.SUM))

        for _ in range(60):
            if not hi - lo > 0.0:
                break
            mid = lo + (hi - lo) / 2
            if mid == lo or mid == hi:
                break
            if count_at(mid) >= max_terms:
                lo = mid
            else:
                hi = mid
        st.cutoff(lo if lo != 0.0 else 5e-324)
