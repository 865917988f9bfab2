"""pl_commutator_noalloc: the commutator for callers that cannot let the
library allocate device memory (hosts that own the whole device through
their own pool, callers that cannot afford an allocation's synchronisation).

Its scratch is a static device array inside libpaulib_b200.so; the caller
passes only inputs and outputs.  The result must equal the allocating
pl_commutator's -- same terms, same deterministic order, same values -- on
two calls in a row (the second call reuses the array the first one left
behind).  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(entry, a, b, mul_i, cap):
    import torch
    from paulib_b200 import _abi
    da = _abi.DeviceSum.from_host(a.x, a.z, a.flags, a.val)
    db = _abi.DeviceSum.from_host(b.x, b.z, b.flags, b.val)
    out = _abi.DeviceSum(a.array_size, cap)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    _abi.check(entry(a.array_size, mul_i, *da.ptrs(), a.n, *db.ptrs(), b.n, *out.ptrs(), cap,
                     cnt.data_ptr(), _abi.stream_ptr()))
    torch.cuda.synchronize()
    n = int(cnt.item())
    return n, out.to_host(n)


@pytest.mark.parametrize("mul_i", [0, 1])
def test_noalloc_matches_allocating_commutator_twice(cuda, mul_i):
    from paulib_b200 import _abi
    from paulib_b200 import workloads as W
    L = _abi.lib()
    a, b = W.window_sums(seed=6, terms=1500)
    cap = a.n * b.n // 8
    n_ref, ref = _run(L.pl_commutator, a, b, mul_i, cap)
    assert n_ref > 0
    for _ in range(2):
        n, got = _run(L.pl_commutator_noalloc, a, b, mul_i, cap)
        assert n == n_ref
        for g, r in zip(got[:3], ref[:3]):  # x, z, flags: exact
            assert np.array_equal(g, r)
        # deterministic and exact; any tolerance would also hold (1e-12 relative)
        assert np.array_equal(got[3].view(np.uint64), ref[3].view(np.uint64))


def test_noalloc_rejects_oversized_requests(cuda):
    from paulib_b200 import _abi
    L = _abi.lib()
    dummy = ctypes.c_void_p(1)
    args = [dummy] * 4
    # 2^15 x 2^15 = 2^30 pairs > 2^29: rejected before any device work
    rc = L.pl_commutator_noalloc(1, 0, *args, 1 << 15, *args, 1 << 15, *args, 1, dummy, None)
    assert rc == _abi.PL_ERR_INVALID_ARG
    assert b"2^29" in L.pl_last_error_message()


def test_noalloc_accepts_exactly_the_limit(cuda):
    # 2^15 x 2^14 = 2^29 pairs fill the static array's 2^16 look-back tiles
    # exactly.  All-Z strings commute pairwise, so nothing is emitted and no
    # output memory is needed.  One more rhs term is over the limit.
    import torch
    from paulib_b200 import _abi
    from paulib_b200.planes import Planes
    L = _abi.lib()
    rng = np.random.default_rng(3)

    def all_z(n):
        z = rng.integers(1, 1 << 20, size=(1, n), dtype=np.uint64)
        return Planes(np.zeros((1, n), np.uint64), z, np.zeros(n, np.uint8),
                      rng.standard_normal(n))

    a, b = all_z(1 << 15), all_z((1 << 14) + 1)
    da = _abi.DeviceSum.from_host(a.x, a.z, a.flags, a.val)
    db = _abi.DeviceSum.from_host(b.x, b.z, b.flags, b.val)
    out = _abi.DeviceSum(1, 1)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for _ in range(2):
        cnt.zero_()
        rc = L.pl_commutator_noalloc(1, 0, *da.ptrs(), a.n, *db.ptrs(), 1 << 14, *out.ptrs(),
                                     0, cnt.data_ptr(), _abi.stream_ptr())
        assert rc == _abi.PL_OK
        torch.cuda.synchronize()
        assert int(cnt.item()) == 0
    rc = L.pl_commutator_noalloc(1, 0, *da.ptrs(), a.n, *db.ptrs(), (1 << 14) + 1, *out.ptrs(),
                                 0, cnt.data_ptr(), _abi.stream_ptr())
    assert rc == _abi.PL_ERR_INVALID_ARG
