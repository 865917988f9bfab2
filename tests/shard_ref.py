"""Test-side restatement of the sharded layout (MpiPauliSum.h:72-84,
101-140): FNV-1a owner of a term and the per-owner buckets in term order, as
term records (x words, z words, flags, value bits)."""
import numpy as np

FNV_OFFSET = 0xcbf29ce484222325
FNV_PRIME = 0x100000001b3
MASK = (1 << 64) - 1


def owners(x, z, ranks):
    aw, n = x.shape
    out = np.empty(n, np.int64)
    for i in range(n):
        h = FNV_OFFSET
        for k in range(aw):
            h = ((h ^ int(x[k, i])) * FNV_PRIME) & MASK
            h = ((h ^ int(z[k, i])) * FNV_PRIME) & MASK
        out[i] = h % ranks
    return out


def records(x, z, f, v):
    aw, n = x.shape
    r = np.empty((n, 2 * aw + 2), np.uint64)
    r[:, :aw] = x.T
    r[:, aw:2 * aw] = z.T
    r[:, 2 * aw] = f.astype(np.uint64)
    r[:, 2 * aw + 1] = np.ascontiguousarray(v, np.float64).view(np.uint64)
    return r


def pack(x, z, f, v, ranks):
    """(records grouped by owner in term order, counts per owner)."""
    o = owners(x, z, ranks)
    rec = records(x, z, f, v)
    order = np.argsort(o, kind="stable")
    return rec[order], np.bincount(o, minlength=ranks)
