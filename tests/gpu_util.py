"""Device-side helpers for the GPU parity tests (calls go through the C ABI)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from paulib_b200.planes import Planes
from paulib_b200 import _abi


def dev(p: Planes, capacity=None) -> _abi.DeviceSum:
    return _abi.DeviceSum.from_host(p.x, p.z, p.flags, p.val, capacity)


def host(ds: _abi.DeviceSum, n=None) -> Planes:
    x, z, f, v = ds.to_host(n)
    return Planes(x, z, f, v)


def gpu_multiply(a: Planes, b: Planes, dropin=False) -> Planes:
    import torch
    L = _abi.lib()
    da, db = dev(a), dev(b)
    out = _abi.DeviceSum(a.array_size, a.n * b.n)
    s = _abi.stream_ptr()
    if dropin:
        L.launch_gpu_mul_soa(a.array_size, *da.ptrs(), *db.ptrs(), *out.ptrs(), a.n, b.n, s)
        _abi.check(_abi.last_error(), "launch_gpu_mul_soa")
    else:
        _abi.check(L.pl_multiply(a.array_size, *da.ptrs(), a.n, *db.ptrs(), b.n, *out.ptrs(), s),
                   "pl_multiply")
    torch.cuda.synchronize()
    out.n = a.n * b.n
    return host(out)


def gpu_commutator(a: Planes, b: Planes, mul_i=False, capacity=None, dropin=False) -> Planes:
    import torch
    L = _abi.lib()
    da, db = dev(a), dev(b)
    cap = a.n * b.n if capacity is None else capacity
    out = _abi.DeviceSum(a.array_size, cap)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = _abi.stream_ptr()
    if dropin:
        L.launch_gpu_commutator_soa(a.array_size, int(mul_i), *da.ptrs(), *db.ptrs(),
                                    *out.ptrs(), cnt.data_ptr(), a.n, b.n, cap, s)
        torch.cuda.synchronize()
        _abi.check(_abi.last_error(), "launch_gpu_commutator_soa")
    else:
        _abi.check(L.pl_commutator(a.array_size, int(mul_i), *da.ptrs(), a.n, *db.ptrs(), b.n,
                                   *out.ptrs(), cap, cnt.data_ptr(), s), "pl_commutator")
    torch.cuda.synchronize()
    out.n = int(cnt.item())
    return host(out)


def _opts(mode, cutoff=0.0, max_weight=None):
    return _abi.CollateOpts(mode, 0, float(cutoff),
                            _abi.UINT64_MAX if max_weight is None else int(max_weight))


def gpu_collate(p: Planes, mode=_abi.PL_COLLATE_CANONICALIZE, cutoff=0.0, max_weight=None,
                capacity=None) -> Planes:
    L = _abi.lib()
    d = dev(p)
    cap = p.n if capacity is None else capacity
    out = _abi.DeviceSum(p.array_size, cap)
    nb = C.c_size_t()
    _abi.check(L.pl_collate_workspace_size(p.array_size, p.n, C.byref(nb)))
    ws = _abi.workspace(nb.value)
    cnt = C.c_int64()
    opts = _opts(mode, cutoff, max_weight)
    _abi.check(L.pl_collate(p.array_size, *d.ptrs(), p.n, *out.ptrs(), cap, C.byref(cnt),
                            C.byref(opts), ws.data_ptr(), nb.value, _abi.stream_ptr()),
               "pl_collate")
    out.n = cnt.value
    return host(out)


def gpu_multiply_collate(a: Planes, b: Planes, mode=_abi.PL_COLLATE_CANONICALIZE, cutoff=0.0,
                         max_weight=None, capacity=None) -> Planes:
    L = _abi.lib()
    da, db = dev(a), dev(b)
    cap = a.n * b.n if capacity is None else capacity
    out = _abi.DeviceSum(a.array_size, cap)
    nb = C.c_size_t()
    _abi.check(L.pl_multiply_collate_workspace_size(a.array_size, a.n, b.n, C.byref(nb)))
    ws = _abi.workspace(nb.value)
    cnt = C.c_int64()
    opts = _opts(mode, cutoff, max_weight)
    _abi.check(L.pl_multiply_collate(a.array_size, *da.ptrs(), a.n, *db.ptrs(), b.n,
                                     *out.ptrs(), cap, C.byref(cnt), C.byref(opts),
                                     ws.data_ptr(), nb.value, _abi.stream_ptr()),
               "pl_multiply_collate")
    out.n = cnt.value
    return host(out)


def gpu_cnot(p: Planes, c: int, t: int) -> Planes:
    import torch
    d = dev(p)
    _abi.check(_abi.lib().pl_apply_cnot(p.array_size, d.x.data_ptr(), d.z.data_ptr(),
                                        d.flags.data_ptr(), p.n, d.capacity, c, t,
                                        _abi.stream_ptr()))
    torch.cuda.synchronize()
    return host(d)


def gpu_zero_state(p: Planes) -> float:
    import torch
    d = dev(p)
    r = torch.zeros(1, dtype=torch.float64, device="cuda")
    _abi.check(_abi.lib().pl_zero_state_expectation(p.array_size, d.x.data_ptr(),
                                                    d.flags.data_ptr(), d.val.data_ptr(), p.n,
                                                    d.capacity, r.data_ptr(), _abi.stream_ptr()))
    return float(r.item())


def as_planes(s) -> Planes:
    return Planes(s.x, s.z, s.flags, s.val)
