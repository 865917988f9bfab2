"""Shared helpers for the parity tests."""
from __future__ import annotations

import numpy as np

from paulib_b200.planes import Planes
from paulib_b200 import strings


def planes(terms, words=None) -> Planes:
    x, z, f, v, _ = strings.planes_from_terms(terms, words)
    return Planes(x, z, f, v)


def to_str(p: Planes, nq: int) -> str:
    return strings.get_str(p.x, p.z, p.flags, p.val, nq)


def random_sum(n, words, seed, num_qubits=None, coeffs="signed", flags="random"):
    """random_pauli_sum (PauliSumUtils.h:114-154) with padding bits masked,
    plus the signed non-unit coefficients of the reference tests'
    random_sum_with_coeffs (tests/PauliSumTests.cpp:33-39) or N(0,1)."""
    rng = np.random.default_rng(seed)
    nq = 64 * words if num_qubits is None else num_qubits
    x = rng.integers(0, 2**63, size=(words, n), dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=(words, n), dtype=np.uint64)
    z = rng.integers(0, 2**63, size=(words, n), dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=(words, n), dtype=np.uint64)
    full, rem = divmod(nq, 64)
    for w in range(words):
        if w > full or (w == full and rem == 0):
            x[w] = 0
            z[w] = 0
        elif w == full:
            mask = np.uint64((1 << rem) - 1)
            x[w] &= mask
            z[w] &= mask
    f = rng.integers(0, 4, size=n, dtype=np.uint8) if flags == "random" else np.zeros(n, np.uint8)
    if coeffs == "signed":
        v = np.array([(-1.0 if i % 2 else 1.0) * (0.5 + i) for i in range(n)])
    elif coeffs == "normal":
        v = rng.standard_normal(n)
    else:
        v = np.ones(n)
    return Planes(x, z, f, v)


def key_bytes(p: Planes, i: int, phase_only=False) -> bytes:
    f = int(p.flags[i]) & (1 if phase_only else 3)
    return p.x[:, i].tobytes() + p.z[:, i].tobytes() + bytes([f])


def abs_scale(o, inp: Planes) -> dict:
    """Sum of |contribution| per canonical key (x, z, phase), computed with
    the oracle on |values|: the scale against which a canonicalized
    coefficient's rounding error is judged."""
    q = Planes(inp.x, inp.z, inp.flags & np.uint8(1), np.abs(inp.val))
    c = o.sort_and_combine(q)
    return {key_bytes(c, i): float(c.val[i]) for i in range(c.n)}


def assert_keys_equal(a: Planes, b: Planes):
    assert a.n == b.n, f"term count {a.n} vs {b.n}"
    assert np.array_equal(a.x, b.x), "x planes differ"
    assert np.array_equal(a.z, b.z), "z planes differ"
    assert np.array_equal(a.flags, b.flags), "flags differ"


def assert_values_close(a: Planes, b: Planes, scale=None, rtol=1e-12):
    """|a - b| <= rtol * max(|b|, scale[key]) elementwise."""
    if scale is None:
        ref = np.abs(b.val)
    else:
        ref = np.array([max(abs(float(b.val[i])), scale.get(key_bytes(b, i, True), 0.0))
                        for i in range(b.n)])
    err = np.abs(a.val - b.val)
    bad = err > rtol * ref
    assert not bad.any(), (f"{int(bad.sum())} coefficients differ beyond {rtol} relative; "
                           f"worst {float((err / np.maximum(ref, 1e-300)).max()):.3e}")


def bit_identical(a: Planes, b: Planes) -> bool:
    return a.val.shape == b.val.shape and np.array_equal(a.val.view(np.uint64),
                                                         b.val.view(np.uint64))


def key_records(p: Planes, phase_only=True) -> np.ndarray:
    """One fixed-width byte record per term whose byte order is the sort
    order of the canonical key (x[0..AS), z[0..AS), flags): each u64 word
    big-endian, then the flags byte (its phase bit with phase_only)."""
    aw, n = p.array_size, p.n
    rec = np.empty((n, 16 * aw + 1), np.uint8)
    for k in range(aw):
        rec[:, 8 * k: 8 * k + 8] = np.ascontiguousarray(p.x[k]).astype(">u8").view(
            np.uint8).reshape(n, 8)
        rec[:, 8 * (aw + k): 8 * (aw + k) + 8] = np.ascontiguousarray(p.z[k]).astype(
            ">u8").view(np.uint8).reshape(n, 8)
    rec[:, 16 * aw] = p.flags & np.uint8(1 if phase_only else 3)
    return rec.view(f"V{16 * aw + 1}").ravel()


def assert_values_close_sorted(a: Planes, b: Planes, scale: Planes, rtol=1e-12):
    """Vectorised assert_values_close for canonical sums: `scale` is the
    sort_and_combine of the input with |values| and the sign folded (keys a
    sorted superset of b's keys); |a - b| <= rtol * max(|b|, scale[key])."""
    kb, ks = key_records(b), key_records(scale)
    pos = np.searchsorted(ks, kb)
    assert (pos < ks.shape[0]).all() and (ks[np.minimum(pos, ks.shape[0] - 1)] == kb).all(), \
        "scale keys do not cover the result"
    ref = np.maximum(np.abs(b.val), scale.val[pos])
    err = np.abs(a.val - b.val)
    bad = err > rtol * ref
    assert not bad.any(), (f"{int(bad.sum())} coefficients differ beyond {rtol} relative; "
                           f"worst {float((err / np.maximum(ref, 1e-300)).max()):.3e}")
